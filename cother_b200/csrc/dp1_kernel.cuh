// Phase-1 DP stage interface.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "layout.h"

namespace cbp {

// phase-1 result of one profile (the fields of TDP2OutputAlnData up to
// nTDP2OutputPhase1, src/libmycu/cuss/CuBatchSS_com.h:45-52)
struct Dp1Rec {
    float score;    // alignment score incl. correlation bonus
    float psts;     // number of positive substitution scores on the path
    uint32_t beg;   // beginning coordinates (x<<16)|y, 1-based
    uint32_t end;   // end coordinates (x<<16)|y, 0-based
    int passed;     // score > threshold
};

struct Dp1Args {
    const float* scores = nullptr;   // slab score matrix [Lq][ld]
    long long ld = 0;
    int Lq = 0;
    const float* qtrn = nullptr;     // query transitions [7][Lq+1]
    ProfilesDev db;
    long long col0 = 0;              // first chunk position of the slab
    int p0 = 0;                      // first chunk profile of the slab
    int nprof = 0;                   // profiles in the slab
    uint8_t* btck = nullptr;         // [Lq][ld]
    float* bandbuf = nullptr;        // [5][ld]: the bottom row of a band, for the next
    float* maxsc = nullptr;          // [nprof]
    uint32_t* maxcoords = nullptr;   // [nprof]
    Dp1Rec* recs = nullptr;          // [nprof]
    int warps = 2;                   // warps (profiles) per block of dp1_kernel: 1 or 2
    int* err = nullptr;              // set to 1 when a staging wait gave up (may be null)
    // backtrack codes are computed for the profiles whose maximum exceeds
    // code_thld (the finalization's threshold: it backtraces only those);
    // -inf: for every profile
    float code_thld = -INFINITY;
};

// Phase-1 DP of the slab's profiles; returns the number of kernel launches:
// with a finite code_thld a launch without backtrack codes finds every
// profile's maximum and a second one sweeps the candidates again with codes
// (2), with code_thld = -inf the second alone, for all profiles (1).
int launch_dp1(const Dp1Args& a, cudaStream_t stream);
// Per device, before the first launch_dp1 with two warps per block (and
// outside any stream capture): the shared-memory opt-in of the DP kernels.
void dp1_set_attributes();
void launch_dp1_finalize(const Dp1Args& a, float thld, cudaStream_t stream);
void launch_pass_compact(const Dp1Args& a, int* pass_idx, long long* pass_dst, int* npass,
                         long long* npos, cudaStream_t stream);

}  // namespace cbp
