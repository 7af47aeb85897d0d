// gpufft-b200: asynchronous bulk copies (the TMA unit's untiled cp.async.bulk)
// into shared memory, completed on an mbarrier, with bounded waits.
//
// A bulk copy is issued by one thread and moved by the TMA unit, not by the
// load/store pipe: a 16 KB tile costs one instruction instead of 1024
// eight-byte loads spread over the CTA. No copy here uses .multicast::cluster.
//
// Every wait is bounded (WAIT_LIMIT_NS of wall time read from %globaltimer,
// and WAIT_MAX_POLLS polls). A wait that runs out returns false: the kernel
// then stops issuing copies, drains the copies it already issued (again with
// a bounded wait) and returns, reporting the timeout to the host through a
// flag of its own. Nothing here traps or spins without a limit.
#pragma once

#include "gf_common.cuh"

namespace gfb
{

constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull; // 2 s
constexpr unsigned WAIT_MAX_POLLS = 1u << 25;               // with __nanosleep(64): > 2 s as well

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
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

// Order this thread's earlier view of shared memory (and, through a preceding
// barrier, the other threads' reads of it) before later async-proxy writes.
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

// Wait for the phase of parity `parity` of the barrier to complete; false if it
// did not within `limit_ns` (or WAIT_MAX_POLLS polls).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns = WAIT_LIMIT_NS)
{
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned i = 0; i < WAIT_MAX_POLLS; i++)
    {
        if (mbar_test(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
        __nanosleep(64);
    }
    return false;
}

// Barrier over the 128 threads of named barrier `id` that also returns
// whether any of them passed `v` true (bar.red.or).
__device__ __forceinline__ bool bar_any(int id, int nthreads, bool v)
{
    unsigned r;
    asm volatile("{\n\t.reg .pred p, q;\n\t"
                 "setp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.or.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((unsigned)v), "r"(id), "r"(nthreads)
                 : "memory");
    return r != 0;
}

__device__ __forceinline__ void bar_named(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

} // namespace gfb
