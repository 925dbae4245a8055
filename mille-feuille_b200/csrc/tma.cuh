// tma.cuh -- bulk asynchronous copies (TMA, non-tensor form) and mbarrier
// helpers for sm_100a.  Only local global memory is ever copied (no cluster
// multicast): a CTA stages its own chunk of the matrix into its own shared
// memory.
#pragma once
#include <cstdint>

#include "mf_common.cuh"

namespace mf {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Bulk copy global -> shared (this CTA), completion counted on `bar`.
// dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// L2 policy for data read once per pass (the streamed matrix): evicted
// first, so that the gathered vectors stay resident in L2.
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, unsigned bytes, uint64_t *bar, uint64_t pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait with a suspend-time hint: the thread sleeps until the phase
// completes or about `hint_ns` nanoseconds pass, instead of polling (idle
// warps then take no issue slots from the working ones).
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, unsigned parity, unsigned hint_ns)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait that sleeps between tries (mbar_try_wait_sleep, then
// __nanosleep(backoff_ns) before each retry when backoff_ns > 0); false (and
// status set) when the budget ran out.
__device__ __forceinline__ bool mbar_wait_sleep_bounded(uint64_t *bar, unsigned parity, int *status,
                                                        unsigned long long budget_ns, unsigned backoff_ns = 0)
{
    if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (backoff_ns) __nanosleep(backoff_ns);
        if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
        if (globaltimer_ns() - t0 > budget_ns) {
            atomicCAS(status, DEV_OK, DEV_TIMEOUT);
            return false;
        }
    }
}

// Bounded wait for phase `parity` of `bar`; false (and status set) when the
// budget ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *status,
                                                  unsigned long long budget_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > budget_ns) {
            atomicCAS(status, DEV_OK, DEV_TIMEOUT);
            return false;
        }
    }
}

// Failure paths: waits for copies known to be in flight before a CTA
// leaves.  Bounded, but never shorter than one second, so that a tiny wait
// budget given to a solve cannot let a CTA leave while bulk copies are still
// landing in its shared memory.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, unsigned parity, int *status, unsigned long long budget_ns)
{
    mbar_wait_bounded(bar, parity, status, budget_ns > 1000000000ull ? budget_ns : 1000000000ull);
}

}  // namespace mf
