// Tensor-core form of the profile-profile term.
//
// The reference sums, for each cell, the 20 quotients
// q_a * d_a / (0.5 * (qbg_a + dbg_a)) on CUDA cores
// (src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:159-186). The background of
// a database profile is the same at all its positions, so the sum is a dot
// product of the query position's target frequencies with the database
// position's frequencies divided by the mean background: for one query, the
// whole slab's sums are one GEMM [Lq x 20] x [20 x ncols] (K padded to 32).
// It runs on the tensor cores through cuBLAS with FP32 accumulation; the
// operands are split into a high and a low part (BF16 + BF16 or TF32 +
// TF32) and the product is hi*hi + hi*lo + lo*hi, which keeps the sums
// within about 1e-6 relative of the FP32 form. The sums land in the score
// buffer, where the score kernel reads them in place of its own loop.
#include <cublas_v2.h>
#include <cuda_bf16.h>

#include <string>

#include "cother_b200.h"
#include "common.cuh"
#include "tc_kernel.cuh"

namespace cbp {

namespace {

constexpr int kK = 32;   // contraction length: 20 amino acids, zero padded

__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// one thread per (position, k): query rows, or the slab's database positions
// scaled by 1 / mean background
template <bool kBf16>
__global__ void tc_operands_kernel(const TcArgs a, bool query, void* hi, void* lo)
{
    const long long n = query ? a.Lq : a.ncols;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kK) return;
    const long long pos = i / kK;
    const int k = (int)(i - pos * kK);
    float x = 0.0f;
    if (k < kNAA) {
        if (query) {
            x = a.q.tf[(long long)k * a.q.N + pos];
        } else {
            const long long g = a.col0 + pos;
            const int p = a.db.pro[g];
            const float den = 0.5f * (a.q.bkg[k] + a.db.bkg[(long long)k * a.db.P + p]);
            x = __fdiv_rn(a.db.tf[(long long)k * a.db.N + g], den);
        }
    }
    if (kBf16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        static_cast<__nv_bfloat16*>(hi)[i] = h;
        static_cast<__nv_bfloat16*>(lo)[i] = __float2bfloat16_rn(x - __bfloat162float(h));
    } else {
        const float h = to_tf32(x);
        static_cast<float*>(hi)[i] = h;
        static_cast<float*>(lo)[i] = x - h;
    }
}

void check_cublas(cublasStatus_t st, const char* what)
{
    if (st != CUBLAS_STATUS_SUCCESS)
        throw Error(CBP_ERR_CUDA, std::string("cuBLAS ") + what + " failed (status " +
                                      std::to_string((int)st) + ")");
}

}  // namespace

size_t tc_operand_bytes(int form, long long rows)
{
    return (size_t)rows * kK * (form == CBP_TC_BF16X3 ? 2 : 4);
}

void tc_profile_sums(const TcArgs& a, int form, cublasHandle_t h, void* qhi, void* qlo, void* dhi,
                     void* dlo, float* out, cudaStream_t stream)
{
    if (a.ncols <= 0 || a.Lq <= 0) return;
    const bool bf = (form == CBP_TC_BF16X3);
    const int threads = 256;
    for (int query = 0; query < 2; query++) {
        const long long n = (query ? a.Lq : a.ncols) * (long long)kK;
        const unsigned blocks = (unsigned)ceil_div(n, threads);
        void* hi = query ? qhi : dhi;
        void* lo = query ? qlo : dlo;
        if (bf) tc_operands_kernel<true><<<blocks, threads, 0, stream>>>(a, query != 0, hi, lo);
        else tc_operands_kernel<false><<<blocks, threads, 0, stream>>>(a, query != 0, hi, lo);
        CBP_CHECK_LAUNCH();
    }
    // column-major view: out[ncols x Lq] (ld a.ld) = D^T (ncols x 32) * Q (32 x Lq),
    // i.e. the row-major [Lq][ld] score layout
    check_cublas(cublasSetStream(h, stream), "set stream");
    const cudaDataType_t t = bf ? CUDA_R_16BF : CUDA_R_32F;
    const cublasComputeType_t ct = bf ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_32F_FAST_TF32;
    const float one = 1.0f, zero = 0.0f;
    const int m = a.ncols, n = a.Lq;
    const void* A[3] = {dhi, dhi, dlo};
    const void* B[3] = {qhi, qlo, qhi};
    for (int k = 0; k < 3; k++)
        check_cublas(cublasGemmEx(h, CUBLAS_OP_T, CUBLAS_OP_N, m, n, kK, &one, A[k], t, kK, B[k], t,
                                  kK, k == 0 ? &zero : &one, out, CUDA_R_32F, (int)a.ld, ct,
                                  CUBLAS_GEMM_DEFAULT),
                     "GEMM");
}

}  // namespace cbp
