// Tensor-core form of the profile-profile term: interface.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include "layout.h"

namespace cbp {

struct TcArgs {
    ProfilesDev q;        // query profile
    ProfilesDev db;       // resident database chunk
    long long col0 = 0;   // first chunk position of the slab
    int ncols = 0;        // slab positions
    long long ld = 0;     // leading dimension of the score matrix
    int Lq = 0;
};

// bytes of one operand (high or low part) for `rows` positions
size_t tc_operand_bytes(int form, long long rows);

// The profile-profile sums of the slab into out ([Lq][ld]): operand
// preparation kernels and three cuBLAS GEMMs on `stream`.
void tc_profile_sums(const TcArgs& a, int form, cublasHandle_t h, void* qhi, void* qlo, void* dhi,
                     void* dlo, float* out, cudaStream_t stream);

}  // namespace cbp
