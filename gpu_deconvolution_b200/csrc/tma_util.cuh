// Bulk asynchronous copies (TMA, cp.async.bulk) and mbarrier helpers for
// sm_100a.  Every wait is bounded: after max_spins polls it gives up and the
// caller records an error status instead of hanging the GPU.
#pragma once

#include <stdint.h>

namespace fmvd {

__device__ __forceinline__ uint32_t smem_u32addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's earlier shared-memory accesses before bulk copies it
// issues afterwards (generic and asynchronous proxy).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32addr(bar)), "r"(bytes)
                 : "memory");
}

// Global -> shared bulk copy completing on bar; dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32addr(bar))
                 : "memory");
}

// Asks the bulk-copy engine to bring [src, src + bytes) into L2 (no
// completion to wait for); src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the given phase parity; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int max_spins = 1 << 22)
{
    for (int i = 0; i < max_spins; i++) {
        if (mbar_try_wait(bar, parity))
            return true;
        if (i > 32)
            __nanosleep(64);
    }
    return false;
}

} // namespace fmvd
