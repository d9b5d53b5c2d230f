// Bulk asynchronous copies (cp.async.bulk, the TMA unit's untiled form) into
// shared memory, completed through a transaction-count mbarrier, for sm_100a.
// Every wait is bounded: a wait that runs out sets a bit in a device status
// word the host reads (IBLGF_ETIMEOUT) instead of spinning for ever.
#pragma once
#include <cuda_runtime.h>

namespace iblgf_b200
{
// iterations of mbarrier.try_wait (each suspends the thread for a
// hardware-defined interval) before a wait counts as timed out
constexpr long long kWaitLimit = 1LL << 22;
constexpr int kStatusTimeout = 1;

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of bulk-copy transactions
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// one plain arrival
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity; false if it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit = kWaitLimit)
{
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// orders this thread's earlier generic-proxy shared-memory accesses (after
// a block barrier: every thread's) before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
}  // namespace iblgf_b200
