// On-device ordering of the reported hits (the top-k hit reduction).
//
// The reference's finalizer keeps the records whose log E-value is at most
// the threshold and that were realigned, and sorts them by log E-value on
// the host (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:79-92,
// src/libmycu/cupro/CuBatchProcessingFinalizer.cpp:276-292). Here every
// slab's records get a 64-bit key on the device as soon as the slab's
// phase 2 is done: the log E-value mapped to an unsigned integer of the
// same order in the high word, the record's index over all slabs in the low
// word, or all ones for a record that is not reported. One bitonic sort
// over all keys of the query then gives the reported hits in the
// finalizer's order -- smallest log E first, equal values in record
// (database) order -- followed by the unreported ones, so any prefix is the
// top k. Only the reported prefix goes back to the host.
#include <cstdint>

#include "common.cuh"
#include "hits_kernel.cuh"
#include "stats_kernel.cuh"

namespace cbp {

namespace {

constexpr int kSortBlock = 4096;      // keys sorted in shared memory by one block
constexpr int kSortThreads = 1024;
constexpr uint64_t kNotReported = ~0ull;

// an unsigned integer of the same order as the float (-0 taken as +0)
__device__ __forceinline__ uint32_t ordered_bits(float f)
{
    if (f == 0.0f) f = 0.0f;
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(256)
hit_keys_kernel(const float* __restrict__ recs, int n, float logethld, long long base, uint64_t* __restrict__ keys,
                int* __restrict__ nreported)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = recs + (long long)i * kRecFloats;
    const float logE = r[rEvalue];
    const int alnlen = __float_as_int(r[rEpA]);   // the phase-2 finalizer's alignment length
    const bool rep = (logE <= logethld) && alnlen >= 1;
    keys[base + i] = rep ? (((uint64_t)ordered_bits(logE) << 32) | (uint64_t)(base + i)) : kNotReported;
    if (rep) atomicAdd(nreported, 1);
}

__global__ void __launch_bounds__(256)
fill_kernel(uint64_t* __restrict__ keys, long long from, long long to)
{
    const long long i = from + blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < to) keys[i] = kNotReported;
}

// Bitonic stages k = kmin .. kmax (powers of two) inside blocks of
// kSortBlock keys, each stage with its distances j = min(k/2, kSortBlock/2)
// .. 1; element i of the sequence sorts ascending when (i & k) == 0.
__global__ void __launch_bounds__(kSortThreads)
bitonic_local(uint64_t* __restrict__ keys, long long kmin, long long kmax)
{
    __shared__ uint64_t s[kSortBlock];
    const long long base = (long long)blockIdx.x * kSortBlock;
    for (int i = threadIdx.x; i < kSortBlock; i += kSortThreads) s[i] = keys[base + i];
    __syncthreads();
    for (long long k = kmin; k <= kmax; k <<= 1) {
        for (int j = (int)(k / 2 < kSortBlock / 2 ? k / 2 : kSortBlock / 2); j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < kSortBlock / 2; t += kSortThreads) {
                const int i = 2 * t - (t & (j - 1));   // lower element of the t-th pair
                const int l = i + j;
                const bool up = ((base + i) & k) == 0;
                const uint64_t a = s[i], b = s[l];
                if ((a > b) == up) { s[i] = b; s[l] = a; }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < kSortBlock; i += kSortThreads) keys[base + i] = s[i];
}

// One bitonic stage (k, j) with j >= kSortBlock across the whole sequence.
__global__ void __launch_bounds__(256)
bitonic_global(uint64_t* __restrict__ keys, long long n2, long long k, long long j)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;   // pair index
    if (t >= n2 / 2) return;
    const long long i = 2 * t - (t & (j - 1));
    const long long l = i + j;
    const bool up = (i & k) == 0;
    const uint64_t a = keys[i], b = keys[l];
    if ((a > b) == up) { keys[i] = b; keys[l] = a; }
}

}  // namespace

long long hit_sort_capacity(long long n)
{
    long long n2 = kSortBlock;
    while (n2 < n) n2 <<= 1;
    return n2;
}

int launch_hit_keys(const float* recs, int n, float logethld, long long base, uint64_t* keys, int* nreported,
                    cudaStream_t stream)
{
    if (n <= 0) return 0;
    hit_keys_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, stream>>>(recs, n, logethld, base, keys, nreported);
    CBP_CHECK_LAUNCH();
    return 1;
}

int launch_hit_sort(uint64_t* keys, long long n, cudaStream_t stream)
{
    const long long n2 = hit_sort_capacity(n);
    int launches = 0;
    if (n2 > n) {
        fill_kernel<<<(unsigned)ceil_div(n2 - n, 256), 256, 0, stream>>>(keys, n, n2);
        CBP_CHECK_LAUNCH();
        launches++;
    }
    const unsigned blocks = (unsigned)(n2 / kSortBlock);
    bitonic_local<<<blocks, kSortThreads, 0, stream>>>(keys, 2, kSortBlock);
    CBP_CHECK_LAUNCH();
    launches++;
    for (long long k = 2 * (long long)kSortBlock; k <= n2; k <<= 1) {
        for (long long j = k / 2; j >= kSortBlock; j >>= 1) {
            bitonic_global<<<(unsigned)ceil_div(n2 / 2, 256), 256, 0, stream>>>(keys, n2, k, j);
            CBP_CHECK_LAUNCH();
            launches++;
        }
        bitonic_local<<<blocks, kSortThreads, 0, stream>>>(keys, k, k);
        CBP_CHECK_LAUNCH();
        launches++;
    }
    return launches;
}

}  // namespace cbp
