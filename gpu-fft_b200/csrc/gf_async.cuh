// gpufft-b200: asynchronous bulk copies (the TMA unit's cp.async.bulk) into
// shared memory, completed on an mbarrier, with bounded waits.
//
// Every wait gives up after a fixed number of polls, records the failure in
// g_async_timeout and lets the kernel return, so a lost copy can never hang a
// GPU; gpufft_device_error_flags() reports it on the host.
#pragma once

#include "gf_common.cuh"

namespace gfb
{

// Set by a kernel whose mbarrier wait ran out of polls (defined in gf_status.cu).
extern __device__ unsigned g_async_timeout;

constexpr unsigned MBAR_MAX_POLLS = 1u << 22; // ~ tens of ms at one poll per few hundred ns

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make initialised mbarriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on the barrier and announce `bytes` of asynchronous transactions.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses 16-byte
// aligned) whose completion is counted on `bar`. No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier; false (and the timeout flag set) if
// it did not complete within MBAR_MAX_POLLS polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    for (unsigned i = 0; i < MBAR_MAX_POLLS; i++)
        if (mbar_test(bar, parity)) return true;
    atomicExch(&g_async_timeout, 1u);
    return false;
}

} // namespace gfb
