// Phase-2 MAP stage interface.
#pragma once

#include <cuda_runtime.h>
#include "layout.h"
#include "stats_kernel.cuh"

namespace cbp {

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
    float* fb = nullptr;                // [Lq][ld2] forward+backward log MM
    float* strip = nullptr;             // [5][ld2] band edges
    uint8_t* btck = nullptr;            // [Lq][ld2] MAP backtrack codes
    long long ld2 = 0;
    char* alns = nullptr;               // [5][alnstride] alignment rows
    long long alnstride = 0;
};

void launch_map(const MapArgs& a, cudaStream_t stream);

}  // namespace cbp
