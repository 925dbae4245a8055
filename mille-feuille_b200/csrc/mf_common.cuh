// mf_common.cuh -- shared device/host helpers for the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "mf.h"

#define MF_TILE 16

namespace mf {

// ---------------------------------------------------------------------------
// Host-side error handling: every CUDA call is checked and turned into an
// mf_status; nothing aborts the process.
// ---------------------------------------------------------------------------
void set_last_error(const char *fmt, ...);
// Counts kernel launches issued by the library (mf_kernel_launches()).
void note_launch(int k = 1);
// Stream-ordered temporary allocation from the library's own memory pool of
// the current device (created on first use; it keeps up to 256 MiB of freed
// memory across synchronisations instead of returning it each time, so the
// temporaries of a solve's checkpoints cost no driver allocation).  Free
// with cudaFreeAsync.
cudaError_t pool_malloc_async(void **p, size_t bytes, cudaStream_t s);
template <typename T>
inline cudaError_t pool_malloc_async(T **p, size_t bytes, cudaStream_t s)
{
    return pool_malloc_async((void **)p, bytes, s);
}

#define MF_CUDA(expr)                                                                     \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess) {                                                          \
            ::mf::set_last_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,               \
                                 cudaGetErrorString(_e));                                 \
            return (_e == cudaErrorMemoryAllocation) ? MF_ERR_NO_MEMORY : MF_ERR_CUDA;    \
        }                                                                                 \
    } while (0)

#define MF_TRY(expr)                                                                      \
    do {                                                                                  \
        mf_status _s = (expr);                                                            \
        if (_s != MF_OK) return _s;                                                       \
    } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

#ifndef MF_BARRIER_SLEEP_NS
#define MF_BARRIER_SLEEP_NS 64  // sleep between grid-barrier polls after the first few
#endif

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ int ld_volatile_i32(const int *p)
{
    return *(const volatile int *)p;
}

// Status word codes written by kernels (device side mirror of mf_status).
enum : int { DEV_OK = 0, DEV_TIMEOUT = MF_ERR_TIMEOUT, DEV_BREAKDOWN = MF_ERR_BREAKDOWN };

// Grid-wide barrier for a cooperative launch.  Every CTA calls it with the
// same running `epoch`; the counter is reset to 0 before the launch.  The
// spin is bounded by `budget_ns`: on expiry the status word is set to
// DEV_TIMEOUT and the call returns false (the caller then leaves the kernel).
__device__ __forceinline__ bool grid_barrier(unsigned long long *counter, unsigned long long target,
                                             int *status, unsigned long long budget_ns)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(counter, 1ull);
        unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_u64(counter) < target) {
            if (((++spins) & 63u) == 0u) {
                if (ld_volatile_i32(status) != DEV_OK) { ok = 0; break; }
                if (globaltimer_ns() - t0 > budget_ns) {
                    atomicCAS(status, DEV_OK, DEV_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ld_volatile_i32(status) != DEV_OK) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid-wide barrier with sharded arrival: CTA g arrives on sub-counter
// g % 8 (each on its own 128-byte line); the last arrival of a group bumps
// the top counter, on which every CTA spins.  ctr points at 9 lines
// (ctr[0], ctr[16], ..., ctr[128]), zeroed before the launch.  `epoch` is
// the 1-based count of barriers this launch has passed.
__device__ __forceinline__ bool grid_barrier_sharded(unsigned long long *ctr, unsigned long long epoch, int *status,
                                                     unsigned long long budget_ns)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned G = gridDim.x;
        const unsigned sub = blockIdx.x & 7u;
        const unsigned long long gsize = (G - sub + 7u) / 8u;
        const unsigned long long ng = G < 8u ? G : 8u;
        __threadfence();
        const unsigned long long old = atomicAdd(ctr + 16 * sub, 1ull);
        if (old + 1ull == epoch * gsize) {
            __threadfence();
            atomicAdd(ctr + 128, 1ull);
        }
        unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_u64(ctr + 128) < epoch * ng) {
            if (((++spins) & 63u) == 0u) {
                if (ld_volatile_i32(status) != DEV_OK) { ok = 0; break; }
                if (globaltimer_ns() - t0 > budget_ns) {
                    atomicCAS(status, DEV_OK, DEV_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ld_volatile_i32(status) != DEV_OK) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p, unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

// Grid-wide barrier with sharded arrival and one-way ordering: the arrival
// is an acquire-release atomic (it publishes every write the CTA made before
// the preceding __syncthreads, and the last arrival of a group carries its
// group's writes on to the top counter), the spin is an acquire load.  No
// full fences: one L2 round trip to arrive, one per poll.  Same counters and
// epochs as grid_barrier_sharded.  A CTA that gives up (budget, or another
// CTA's error status seen while spinning) returns false.
__device__ __forceinline__ bool grid_barrier_fast(unsigned long long *ctr, unsigned long long epoch, int *status,
                                                  unsigned long long budget_ns)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned G = gridDim.x;
        const unsigned sub = blockIdx.x & 7u;
        const unsigned long long gsize = (G - sub + 7u) / 8u;
        const unsigned long long ng = G < 8u ? G : 8u;
        const unsigned long long old = atom_add_acq_rel_u64(ctr + 16 * sub, 1ull);
        if (old + 1ull == epoch * gsize) atom_add_acq_rel_u64(ctr + 128, 1ull);
        if (ld_acquire_u64(ctr + 128) < epoch * ng) {
            const unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            while (ld_acquire_u64(ctr + 128) < epoch * ng) {
                if (((++spins) & 31u) == 0u) {
                    if (ld_volatile_i32(status) != DEV_OK) { ok = 0; break; }
                    if (globaltimer_ns() - t0 > budget_ns) {
                        atomicCAS(status, DEV_OK, DEV_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void red_add_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid-wide barrier on one counter: every CTA adds 1 with a release
// reduction (no round trip to wait for) and spins with acquire loads until
// the counter reaches epoch * gridDim.x.  Same bounded-spin and status rules
// as grid_barrier_fast; ctr[0] must be zero at launch.
__device__ __forceinline__ bool grid_barrier_flat(unsigned long long *ctr, unsigned long long epoch, int *status,
                                                  unsigned long long budget_ns)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned long long target = epoch * (unsigned long long)gridDim.x;
        red_add_release_u64(ctr, 1ull);
        if (ld_relaxed_u64(ctr) < target) {
            // relaxed polls (no L1 invalidation each), a short sleep after
            // the first few so that a waiting CTA leaves the issue slots to
            // the CTAs still computing on its SM
            const unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            while (ld_relaxed_u64(ctr) < target) {
                ++spins;
                if (MF_BARRIER_SLEEP_NS > 0 && spins > 8u) __nanosleep(MF_BARRIER_SLEEP_NS);
                if ((spins & 15u) == 0u) {
                    if (ld_volatile_i32(status) != DEV_OK) { ok = 0; break; }
                    if (globaltimer_ns() - t0 > budget_ns) {
                        atomicCAS(status, DEV_OK, DEV_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        fence_acq_rel_gpu();  // with the relaxed load that saw the target: acquire
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Deterministic CTA reduction of one double per thread: warp butterfly, then
// the warp results summed in warp order.  All threads get the result.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *s_warp)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_warp[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) s += s_warp[i];
    return s;
}

// Deterministic sum of `count` per-CTA partials (same order in every CTA):
// lane l sums entries l, l+32, ... sequentially, then a butterfly.
__device__ __forceinline__ double warp_sum_partials(const double *part, int count)
{
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    // batches of 8 independent loads per lane (one L2 round trip per batch)
    for (int i0 = lane; i0 < count; i0 += 32 * 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = i0 + 32 * u;
            v[u] = (i < count) ? __ldcg(part + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) s += v[u];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// Deterministic sum of `count` per-CTA partials by a whole CTA (same order
// in every CTA): thread t sums entries t, t + NT, ... (loads issued four at
// a time: up to 4 NT partials in one L2 round trip), then the fixed block
// tree.  All threads get the result.
template <int NT>
__device__ __forceinline__ double block_sum_partials(const double *part, int count, double *s_warp)
{
    double s = 0.0;
    constexpr int B = 4;
    for (int i0 = threadIdx.x; i0 < count; i0 += NT * B) {
        double v[B];
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int i = i0 + NT * u;
            v[u] = (i < count) ? __ldcg(part + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < B; u++) s += v[u];
    }
    return block_sum<NT>(s, s_warp);
}

}  // namespace mf
