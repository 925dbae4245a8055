// selftest.cu -- exercises the bounded waits of the persistent kernels on a
// condition that never becomes true, so that the timeout path (status word,
// clean return, usable context) is tested without faulting or hanging a GPU.
// No reference counterpart: the reference's spin-waits are unbounded.
#include "mf_internal.h"
#include "tma.cuh"

namespace mf {
namespace {

// Each CTA arrives once at a grid barrier, then waits for a second epoch
// that nobody will complete, then waits on an mbarrier nobody arrives at.
// Both waits must expire after the budget and report DEV_TIMEOUT.
__global__ void k_wait_selftest(unsigned long long *ctr, int *status, unsigned long long budget_ns, int *ok_out)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const bool first = grid_barrier_fast(ctr, 1, status, budget_ns);   // every CTA arrives: completes
    const bool second = grid_barrier_fast(ctr, 3, status, budget_ns);  // epoch 3 is never reached
    // a fresh status for the mbarrier wait (the first expiry set it already)
    __shared__ int local_status;
    if (threadIdx.x == 0) local_status = DEV_OK;
    __syncthreads();
    const bool third = mbar_wait_bounded(&bar, 0u, &local_status, budget_ns);  // no arrival ever
    __syncthreads();
    if (threadIdx.x == 0) {
        ok_out[3 * blockIdx.x + 0] = first ? 1 : 0;
        ok_out[3 * blockIdx.x + 1] = second ? 1 : 0;
        ok_out[3 * blockIdx.x + 2] = (!third && local_status == DEV_TIMEOUT) ? 1 : 0;
    }
}

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" mf_status mf_selftest_bounded_waits(double budget_s, int *results)
{
    if (budget_s <= 0 || budget_s > 10 || !results) return MF_ERR_INVALID_ARG;
    unsigned long long *ctr = nullptr;
    int *d_out = nullptr;
    const int G = 2;
    MF_CUDA(cudaMalloc(&ctr, 9 * 128 + sizeof(int) + sizeof(int) * 3 * G));
    int *status = (int *)((char *)ctr + 9 * 128);
    d_out = status + 1;
    cudaError_t e = cudaMemset(ctr, 0, 9 * 128 + sizeof(int) + sizeof(int) * 3 * G);
    if (e == cudaSuccess) {
        k_wait_selftest<<<G, 64>>>(ctr, status, (unsigned long long)(budget_s * 1e9), d_out);
        note_launch();
        e = cudaGetLastError();
    }
    int h[1 + 3 * G] = {0};
    if (e == cudaSuccess) e = cudaMemcpy(h, status, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(ctr);
    if (e != cudaSuccess) {
        set_last_error("selftest: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    // results: [0] device status word, then per CTA: first barrier passed,
    // second barrier passed (must be 0), mbarrier wait expired with TIMEOUT
    for (int k = 0; k < 1 + 3 * G; k++) results[k] = h[k];
    return MF_OK;
}
