// Statistics stage interface.
#pragma once

#include <cuda_runtime.h>
#include "layout.h"
#include "dp1_kernel.cuh"

namespace cbp {

// floats per hit record: the fields of TDP2OutputAlnData
// (src/libmycu/cuss/CuBatchSS_com.h:45-71)
constexpr int kRecFloats = 18;
enum {
    rScore = 0, rOrgProNo, rProNewDst, rPstvs, rBegCoords, rEndCoords,
    rLmbdEst, rKEst, rEvalue, rEpA, rMin, rMax, rE, rH, rLmbd, rK, rIdnts, rNGaps
};

constexpr int kNNWeights = 93;

struct StatsArgs {
    const float* scores = nullptr;   // slab score matrix [Lq][ld]
    long long ld = 0;
    int Lq = 0;
    long long col0 = 0;
    int p0 = 0;
    ProfilesDev db;
    const int8_t* qaa = nullptr;     // query residues
    float qeno = 0.f;
    int x_uninf = 1;
    const int* pass_idx = nullptr;   // slab profile index per passed pair
    const long long* pass_dst = nullptr;
    const Dp1Rec* recs = nullptr;    // phase-1 records (slab index)
    float* out = nullptr;            // [npass][kRecFloats]
    const float* nnweights = nullptr;
    int ssemodel = 2;
    float searchspace = 0.f;
    float ref_lambda = 0.f, ref_K = 0.f;
    float exp_gapped_lambda = 0.f, exp_gapped_K = 0.f;
    // the precision forms: per pair, the parameter fit in FP64 and in FP32
    // (kFitDoubles each: lambda, K, H, E in FP64, then in FP32); with
    // use_fit64 the E-value and the record take the FP64 fit's parameters
    double* fits = nullptr;
    int use_fit64 = 0;
};

constexpr int kFitDoubles = 8;

void launch_stats(const StatsArgs& a, int npass, cudaStream_t stream);

}  // namespace cbp
