// Device-resident data layout of the search path.
//
// Profiles arrive in the reference's 181-field structure-of-arrays form
// (src/libmycu/cupro/PM2DVectorFields.h:51-87). On upload they are repacked
// once into the layout below, sized for HBM bandwidth rather than for the
// reference's one-buffer-per-field heap:
//
//  * target frequencies   tf   [20][N]    float  (coalesced per letter)
//  * SS probabilities     ss   [3][N]     float
//  * distance lists       dst  [N][128]   uint8  -- element k of the list at
//    byte k (k < 99), saturated at 20; 21 marks "no data" and pads bytes
//    99..127; the list length is kept separately in dstlen [N]. 128 B per
//    position instead of the reference's 400 B of floats.
//  * transitions          trn  [7][N+P]   float  (entry pstart[p]+p is the
//    beginning vector of profile p, entry pstart[p]+p+1+k its position k)
//  * per profile          bkg [20][P], eno [P], plen [P], pstart [P]
//  * per position         pro [N] (profile index), aa [N], sss [N]
#pragma once

#include <stdint.h>

namespace cbp {

constexpr int kNAA = 20;
constexpr int kNCV = 19;          // context-vector entries (pmv2DNoCVEls)
constexpr int kNSS = 3;
constexpr int kNTrn = 7;
constexpr int kMaxDst = 99;
constexpr int kDstStride = 128;     // bytes per position in the packed lists
constexpr int kDstNoData = 21;      // packed code of 255 (no data)
constexpr int kDstCard = 22;        // packed codes 0..21
constexpr int kSSCard = 30;

// transition indices (src/libmycu/cudp/CuBatchDP_com.h:84-93)
enum { trMM = 0, trMI = 1, trMD = 2, trIM = 3, trII = 4, trDM = 5, trDD = 6 };

struct ProfilesDev {
    long long N = 0;        // positions
    int P = 0;              // profiles
    const float* tf = nullptr;
    const float* ss = nullptr;
    const uint8_t* dst = nullptr;
    const uint8_t* dstlen = nullptr;
    const float* trn = nullptr;
    const float* bkg = nullptr;
    const float* eno = nullptr;
    const int* plen = nullptr;
    const long long* pstart = nullptr;
    const int* pro = nullptr;
    const int8_t* aa = nullptr;
    const int8_t* sss = nullptr;
    // context vectors, when uploaded: [19][N] entries, [N] log priors, [N]
    // squared norms
    const float* cv = nullptr;
    const float* cvprior = nullptr;
    const float* cvnorm2 = nullptr;
};

}  // namespace cbp
