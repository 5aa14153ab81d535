// Phase-2 MAP stage interface.
#pragma once

#include <cuda_runtime.h>
#include "layout.h"
#include "stats_kernel.cuh"

namespace cbp {

// Phase-2 matrices of a slab are kept in a skewed band layout over the
// phase-2 column space (the realigned profiles side by side, pass_dst[k]
// the first column of pair k): cell (r, g) lies in band r/32 at diagonal
// row g + r%32, lane r%32, so that the 32 cells a warp visits at one step
// of an anti-diagonal sweep are one contiguous 128-byte row. A band has
// `nd` = phase-2 positions + 31 diagonal rows; neighbouring pairs share
// their first and last 31 rows, in disjoint lanes.
constexpr int kMapMaxWarps = 8;     // warps (32-row bands in flight) per pair
constexpr int kMapEdgeFields = 6;   // floats per column of a band edge

struct MapArgs {
    const float* scores = nullptr;      // slab score matrix [Lq][ld]
    const float* modscores = nullptr;   // slab modular scores [Lq][ld]
    long long ld = 0;
    int Lq = 0;
    long long col0 = 0;
    int p0 = 0;
    ProfilesDev db;
    const float* qtrn = nullptr;        // query transitions [7][Lq+1]
    const int8_t* qaa = nullptr;
    const int8_t* qsss = nullptr;
    int printsss = 1;
    int modscores_inuse = 1;
    float minpp = 0.28f;
    float logevthld = 0.f;
    int npass = 0;
    const int* pass_idx = nullptr;
    const long long* pass_dst = nullptr;   // phase-2 column of each pair
    float* recs = nullptr;              // [npass][kRecFloats], updated in place
    long long nd = 0;                   // diagonal rows per band
    float* cs = nullptr;                // [nb][nd][32] cell scores with the pair's offset/multiplier
    float* fb = nullptr;                // [nb][nd][32] forward, then forward + backward, log MM
    unsigned* sg = nullptr;             // [nb][nd] bit t: raw score of row 32b+t > 0
    unsigned long long* bt = nullptr;   // [nb][nd] MAP backtrack codes: bit t | bit 32+t
    float* strip = nullptr;             // [kMapMaxWarps][6][Ld] band edges per pair, at 48*pass_dst
    int* err = nullptr;                 // set when a wait between warps gives up
    char* alns = nullptr;               // [5][alnstride] alignment rows
    long long alnstride = 0;
};

inline long long map_diag_rows(long long npos2) { return npos2 + 31; }
inline long long map_bands(int Lq) { return (Lq + 31) / 32; }
inline long long map_strip_floats(long long npos2)
{
    return (long long)kMapMaxWarps * kMapEdgeFields * npos2;
}

// zeroes sg and bt, then realigns every pair of the pass list
void launch_map(const MapArgs& a, cudaStream_t stream);

// MAPALN=0: alignment rows and counts of the pass list's pairs from their
// phase-1 backtrack codes ([Lq][ld] of the slab), starting at the phase-1
// maximum (maxsc1/maxcoords1 per slab profile). Uses the slab, query,
// pass-list, record and alignment-row fields of `a`, not the phase-2
// buffers.
void launch_aln_final(const MapArgs& a, const uint8_t* btck1, const float* maxsc1,
                      const uint32_t* maxcoords1, cudaStream_t stream);

}  // namespace cbp
