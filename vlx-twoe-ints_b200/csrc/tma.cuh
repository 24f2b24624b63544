// Bulk copies global -> shared memory through the TMA engine (sm_90+ PTX),
// tracked by mbarriers with transaction counts.
//
// Only the plain, non-multicast form is used: cp.async.bulk with a
// shared::cluster destination that is this CTA's own shared memory (every
// CTA is a cluster of one without a cluster launch) and a source in this
// GPU's global memory.  A copy needs a 16-byte aligned source and
// destination and a byte count that is a multiple of 16.
//
// Every wait is bounded: tma_wait gives up after TMA_WAIT_LIMIT polls and
// reports it, so a copy that never lands ends the kernel with an error flag
// instead of a hang.
#pragma once
#include <stdint.h>

namespace vlxb {

constexpr uint32_t TMA_WAIT_LIMIT = 1u << 24;  // polls of try_wait (each may suspend briefly)

// Error flags of the device error word (vlxb_kernelErrors).
constexpr unsigned long long VLXB_KERR_TMA_TIMEOUT = 1ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the TMA (async) proxy.
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transactions for this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst (shared) <- src (global), `bytes` bytes, completion counted on bar.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; false after
// TMA_WAIT_LIMIT polls.
__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t it = 0; it < TMA_WAIT_LIMIT; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace vlxb
