// 1-D bulk copies (the TMA engine's cp.async.bulk) into shared memory with
// an mbarrier, and a wait that gives up after a time limit. Sources are
// always this GPU's own global memory; no multicast.
#pragma once

#include <cstdint>

namespace cbp {

static __device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
static __device__ __forceinline__ void mbar_init(unsigned long long* b)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(b)) : "memory");
}
// make the initialised mbarrier visible to the bulk-copy (async) proxy
static __device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// the single arrival of the phase, announcing `bytes` of copies
static __device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16
static __device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* b)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(b)) : "memory");
}
static __device__ __forceinline__ bool mbar_test(unsigned long long* b, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
static __device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase of `parity` of an mbarrier to complete, for at most
// limit_ns nanoseconds; false if it did not.
static __device__ __noinline__ bool mbar_wait_for(unsigned long long* b, unsigned parity,
                                                 unsigned long long limit_ns)
{
    if (mbar_test(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(b, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

}  // namespace cbp
