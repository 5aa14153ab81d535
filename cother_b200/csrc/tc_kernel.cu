// Tensor-core form of the profile-profile term, on the 5th-generation
// tensor cores (tcgen05.mma, accumulator in tensor memory).
//
// The reference sums, for each cell, the 20 quotients
// q_a * d_a / (0.5 * (qbg_a + dbg_a)) on CUDA cores
// (src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:159-186). The background of
// a database profile is the same at all its positions, so the sum is a dot
// product of the query position's target frequencies with the database
// position's frequencies divided by the mean background: for one query, a
// slab's sums are the contraction [ncols x 20] . [20 x Lq].
//
// Split precision. Each operand is split into a high and a low part (BF16 +
// BF16, or TF32 + TF32) and the product is hi*hi + hi*lo + lo*hi, which
// keeps the sums within about 1e-6 relative of FP32. The three products are
// one contraction of length 64: the database row is [hi | hi | lo | 0 0 0 0]
// and the query row [hi | lo | hi | 0 0 0 0] (20 + 20 + 20 + 4).
//
// Kernel. Persistent CTAs of 128 threads (three or four per SM) walk tiles
// of 128 database positions (the MMA's M: tensor-memory lanes) by up to 128
// query rows (its N: tensor-memory columns, FP32 accumulator). Per tile:
//  * the database rows are computed in the kernel from the resident
//    frequencies and backgrounds (the split fused in; nothing of it goes
//    through HBM) and stored in shared memory in the MMA's K-major
//    no-swizzle layout: core matrices of 8 rows x 16 bytes, contiguous;
//  * the query rows are a pre-built image of that layout (one small kernel
//    per query), fetched with one bulk copy (cp.async.bulk + mbarrier) and
//    kept while the query tile does not change;
//  * one thread issues the tcgen05.mma chain over K and commits it to an
//    mbarrier;
//  * each warp reads its 32 lanes (database positions) of the accumulator
//    with tcgen05.ld and writes the sums to the [Lq][ld] score buffer: for
//    a fixed query row the warp's 32 lanes are 32 consecutive columns, so
//    every store is one 128-byte line.
// The score kernel then reads the sums in place of its 20-term loop. Every
// wait is bounded (1 s); a wait that gives up flags the launch and the CTA
// releases its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "cother_b200.h"
#include "common.cuh"
#include "tc_kernel.cuh"

namespace cbp {

namespace {

constexpr int kTM = 128;                 // database positions per tile (MMA M)
constexpr int kTNMax = 128;              // query rows per tile (MMA N, at most)
constexpr int kKE = 64;                  // contraction length (3 x 20 + 4 zeros)
constexpr int kThreads = 128;
constexpr int kTmemCols = 128;           // FP32 accumulator columns (four CTAs fill the 512)
constexpr unsigned long long kWaitNs = 1000000000ull;

template <bool kBf16> struct Form {
    static constexpr int kEsz = kBf16 ? 2 : 4;
    static constexpr int kRowBytes = kKE * kEsz;          // 128 or 256
    static constexpr int kCPR = kRowBytes / 16;           // 16-byte chunks per row
    static constexpr int kSBO = kCPR * 128;               // bytes between 8-row groups
    static constexpr int kMmas = kRowBytes / 32;          // K of one MMA is 32 bytes of a row
    static constexpr uint32_t kFmt = kBf16 ? 1u : 2u;     // operand format: BF16 / TF32
    static constexpr int kABytes = kTM * kRowBytes;
    static constexpr int kBBytes = kTNMax * kRowBytes;
    // dynamic shared memory requested per CTA: at most four CTAs per SM
    // (BF16: 32 KB of tiles) or three (TF32: 64 KB), so that their tensor
    // memory (128 columns each) always fits and no allocation waits
    static constexpr size_t kSmemRequest = kBf16 ? 48 * 1024 : 64 * 1024;
    static constexpr int kCtasPerSm = kBf16 ? 4 : 3;
};

// byte offset of 16-byte chunk kc of row r in the no-swizzle K-major layout
template <int kCPR>
__host__ __device__ __forceinline__ int core_offset(int r, int kc)
{
    return ((r >> 3) * kCPR + kc) * 128 + (r & 7) * 16;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading byte offset (the
// next 16-byte column of K), stride byte offset (the next 8 rows), the
// Blackwell descriptor version, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor: FP32 accumulator, A and B of one format, both
// K-major, dense, N x 128
template <bool kBf16>
__device__ __forceinline__ uint32_t instr_desc(int N)
{
    return (1u << 4) | (Form<kBf16>::kFmt << 7) | (Form<kBf16>::kFmt << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(kTM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(unsigned long long* b)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __noinline__ bool mbar_wait(unsigned long long* b, uint32_t parity)
{
    if (mbar_test(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(b, parity))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}

__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// split x into (hi, lo) of the form's type, as 32-bit containers (BF16 in
// the low half)
template <bool kBf16>
__device__ __forceinline__ void split(float x, uint32_t& hi, uint32_t& lo)
{
    if (kBf16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        hi = __bfloat16_as_ushort(h);
        lo = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(h)));
    } else {
        const float h = to_tf32(x);
        hi = __float_as_uint(h);
        lo = __float_as_uint(x - h);
    }
}

// element e (0..63) of an operand row from its 20 split values: the
// database row is hi | hi | lo | 0, the query row hi | lo | hi | 0
__device__ __forceinline__ uint32_t row_elem(const uint32_t* hi, const uint32_t* lo, int e, bool query)
{
    if (e < 20) return hi[e];
    if (e < 40) return query ? lo[e - 20] : hi[e - 20];
    if (e < 60) return query ? hi[e - 40] : lo[e - 40];
    return 0u;
}

// write a row's 64 elements into its 16-byte chunks (dst = chunk 0 of the row)
template <bool kBf16>
__device__ __forceinline__ void store_row(uint8_t* dst, const uint32_t* hi, const uint32_t* lo, bool query)
{
    using F = Form<kBf16>;
#pragma unroll
    for (int kc = 0; kc < F::kCPR; kc++) {
        uint4 v;
        if (kBf16) {
            const int e = kc * 8;
            v.x = row_elem(hi, lo, e + 0, query) | (row_elem(hi, lo, e + 1, query) << 16);
            v.y = row_elem(hi, lo, e + 2, query) | (row_elem(hi, lo, e + 3, query) << 16);
            v.z = row_elem(hi, lo, e + 4, query) | (row_elem(hi, lo, e + 5, query) << 16);
            v.w = row_elem(hi, lo, e + 6, query) | (row_elem(hi, lo, e + 7, query) << 16);
        } else {
            const int e = kc * 4;
            v.x = row_elem(hi, lo, e + 0, query);
            v.y = row_elem(hi, lo, e + 1, query);
            v.z = row_elem(hi, lo, e + 2, query);
            v.w = row_elem(hi, lo, e + 3, query);
        }
        *reinterpret_cast<uint4*>(dst + kc * 128) = v;
    }
}

// The query operand as the shared-memory image of each query tile: tile t
// (rows 128t..128t+127) at t * kBBytes; rows past the query are zero.
template <bool kBf16>
__global__ void __launch_bounds__(128)
tc_query_image_kernel(const TcArgs a, uint8_t* __restrict__ img, int ntiles)
{
    using F = Form<kBf16>;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= ntiles * kTNMax) return;
    uint32_t hi[20], lo[20];
#pragma unroll
    for (int k = 0; k < 20; k++) {
        const float x = r < a.Lq ? a.q.tf[(long long)k * a.q.N + a.qrow0 + r] : 0.0f;
        split<kBf16>(x, hi[k], lo[k]);
    }
    const int t = r / kTNMax, rr = r - t * kTNMax;
    store_row<kBf16>(img + (size_t)t * F::kBBytes + core_offset<F::kCPR>(rr, 0), hi, lo, true);
}

template <bool kBf16>
__global__ void __launch_bounds__(kThreads, 1)
tc_umma_kernel(const TcArgs a, const uint8_t* __restrict__ qimg, float* __restrict__ out, int* __restrict__ err)
{
    using F = Form<kBf16>;
    extern __shared__ __align__(1024) uint8_t s_dyn[];
    uint8_t* sA = s_dyn;
    uint8_t* sB = s_dyn + F::kABytes;
    __shared__ unsigned long long bar_b, bar_mma;
    __shared__ uint32_t s_tmem;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bar_b);
        mbar_init(&bar_mma);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&s_tmem)), "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    const int mtiles = (a.ncols + kTM - 1) / kTM;
    const int ntiles = (a.Lq + kTNMax - 1) / kTNMax;
    uint32_t ph_b = 0, ph_m = 0;
    int loaded = -1;
    bool ok = true;
    for (int mt = blockIdx.x; mt < mtiles && ok; mt += gridDim.x) {
        const long long m0 = (long long)mt * kTM;
        // database rows of the tile: the split computed here
        {
            const long long col = m0 + tid;
            uint32_t hi[20], lo[20];
            if (col < a.ncols) {
                const long long g = a.col0 + col;
                const int p = a.db.pro[g];
#pragma unroll
                for (int k = 0; k < 20; k++) {
                    const float den = 0.5f * (a.q.bkg[(long long)k * a.q.P + a.qprof] +
                                              a.db.bkg[(long long)k * a.db.P + p]);
                    split<kBf16>(__fdiv_rn(a.db.tf[(long long)k * a.db.N + g], den), hi[k], lo[k]);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 20; k++) hi[k] = lo[k] = 0u;
            }
            store_row<kBf16>(sA + core_offset<F::kCPR>(tid, 0), hi, lo, false);
            // the tensor cores read shared memory through the async proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        for (int nt = 0; nt < ntiles && ok; nt++) {
            const int n0 = nt * kTNMax;
            const int nrows = min(kTNMax, a.Lq - n0);
            const int N = (nrows + 15) & ~15;
            if (nt != loaded) {
                if (tid == 0) {
                    const uint32_t bytes = (uint32_t)N * F::kRowBytes;
                    mbar_expect_tx(&bar_b, bytes);
                    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                                 :: "r"(smem_u32(sB)), "l"(qimg + (size_t)nt * F::kBBytes), "r"(bytes),
                                    "r"(smem_u32(&bar_b)) : "memory");
                }
                const bool got = __syncthreads_and(mbar_wait(&bar_b, ph_b));
                if (!got) { ok = false; break; }
                ph_b ^= 1u;
                loaded = nt;
            }
            __syncthreads();     // the database rows are written (and fenced) by every thread
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (tid == 0) {
                const uint32_t idesc = instr_desc<kBf16>(N);
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
                const uint32_t mask = 0u;
#pragma unroll
                for (int s = 0; s < F::kMmas; s++) {
                    const uint64_t da = smem_desc(a0 + 256u * s, 128u, F::kSBO);
                    const uint64_t db = smem_desc(b0 + 256u * s, 128u, F::kSBO);
                    const uint32_t acc = s > 0 ? 1u : 0u;
                    if (kBf16) {
                        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                                     :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask), "r"(mask),
                                        "r"(mask), "r"(mask) : "memory");
                    } else {
                        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                     "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                                     :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask), "r"(mask),
                                        "r"(mask), "r"(mask) : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             :: "r"(smem_u32(&bar_mma)) : "memory");
            }
            const bool done = __syncthreads_and(mbar_wait(&bar_mma, ph_m));
            if (!done) {
                // the MMA did not complete: wait once more (bounded) before
                // the tensor memory is released
                (void)mbar_wait(&bar_mma, ph_m);
                ok = false;
                break;
            }
            ph_m ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // epilogue: lanes 32w..32w+31 of the accumulator are this warp's
            // database positions, columns its query rows
            const long long col = m0 + 32 * warp + lane;
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
            for (int j0 = 0; j0 < N; j0 += 32) {
                // two 16-column loads in flight per wait (N is a multiple of 16)
                uint32_t v[32];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                               "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                             : "r"(taddr + (uint32_t)j0));
                const bool two = j0 + 16 < N;
                if (two)
                    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                                 : "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                                   "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                                 : "r"(taddr + (uint32_t)(j0 + 16)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (col < a.ncols) {
                    float* o = out + (long long)(n0 + j0) * a.ld + col;
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        if (jj >= 16 && !two) break;
                        if (n0 + j0 + jj < a.Lq) o[(long long)jj * a.ld] = __uint_as_float(v[jj]);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();     // the accumulator is read before the next tile's MMA
        }
    }
    if (!ok && tid == 0 && err) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols) : "memory");
}

int sm_count()
{
    int dev = 0, n = 0;
    CBP_CUDA(cudaGetDevice(&dev));
    CBP_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

template <bool kBf16>
int launch_form(const TcArgs& a, void* qimg, float* out, int* err, cudaStream_t stream)
{
    const int ntiles = (int)ceil_div(a.Lq, kTNMax);
    tc_query_image_kernel<kBf16><<<(unsigned)ceil_div((long long)ntiles * kTNMax, 128), 128, 0, stream>>>(
        a, static_cast<uint8_t*>(qimg), ntiles);
    CBP_CHECK_LAUNCH();
    const int mtiles = (int)ceil_div(a.ncols, kTM);
    const int grid = (int)std::min<long long>(mtiles, (long long)Form<kBf16>::kCtasPerSm * sm_count());
    tc_umma_kernel<kBf16><<<grid, kThreads, Form<kBf16>::kSmemRequest, stream>>>(
        a, static_cast<const uint8_t*>(qimg), out, err);
    CBP_CHECK_LAUNCH();
    return 2;
}

}  // namespace

void tc_set_attributes()
{
    CBP_CUDA(cudaFuncSetAttribute(tc_umma_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)Form<true>::kSmemRequest));
    CBP_CUDA(cudaFuncSetAttribute(tc_umma_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)Form<false>::kSmemRequest));
}

size_t tc_query_image_bytes(int form, long long Lq)
{
    const long long ntiles = ceil_div(Lq, kTNMax);
    return (size_t)ntiles * (form == CBP_TC_BF16X3 ? Form<true>::kBBytes : Form<false>::kBBytes);
}

int tc_profile_sums(const TcArgs& a, int form, void* qimg, float* out, int* err, cudaStream_t stream)
{
    if (a.ncols <= 0 || a.Lq <= 0) return 0;
    if (form == CBP_TC_BF16X3) return launch_form<true>(a, qimg, out, err, stream);
    if (form == CBP_TC_TF32X3) return launch_form<false>(a, qimg, out, err, stream);
    throw Error(CBP_ERR_ARG, "unknown tensor-core form");
}

}  // namespace cbp
