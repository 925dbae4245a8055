// scan.cu -- device exclusive prefix sum of int32 arrays (the role of the
// reference's host exclusive_scan, src/utils.h:34-49).  Three phases: block
// totals, a scan of the totals (recursive), then per-block scans with the
// block offset added.  in == out is allowed.
#include "mf_internal.h"

namespace mf {
namespace {

constexpr int SCAN_NT = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_CHUNK = SCAN_NT * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive(int v, int *s_warp, int *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = (lane < SCAN_NT / 32) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < SCAN_NT / 32) s_warp[lane] = t;
    }
    __syncthreads();
    int prefix = (w > 0 ? s_warp[w - 1] : 0) + x - v;
    if (total) *total = s_warp[SCAN_NT / 32 - 1];
    return prefix;
}

__global__ void __launch_bounds__(SCAN_NT) k_block_totals(const int *in, int n, int *totals)
{
    __shared__ int s_warp[SCAN_NT / 32];
    long long base = (long long)blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) sum += in[base + i];
    int tot;
    block_exclusive(sum, s_warp, &tot);
    if (threadIdx.x == 0) totals[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_NT) k_block_scan(const int *in, int *out, int n,
                                                        const int *offsets, int *grand_total)
{
    __shared__ int s_warp[SCAN_NT / 32];
    long long base = (long long)blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        sum += v[i];
    }
    int tot;
    int run = block_exclusive(sum, s_warp, &tot) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_NT - 1) *grand_total = run;
}

mf_status scan_rec(const int *in, int *out, int n, cudaStream_t s, int *d_total)
{
    int blocks = ceil_div(n, SCAN_CHUNK);
    if (blocks <= 1) {
        k_block_scan<<<1, SCAN_NT, 0, s>>>(in, out, n, nullptr, d_total);
        note_launch();
        MF_CUDA(cudaGetLastError());
        return MF_OK;
    }
    int *tot = nullptr;
    MF_CUDA(pool_malloc_async(&tot, sizeof(int) * (blocks + 1), s));
    k_block_totals<<<blocks, SCAN_NT, 0, s>>>(in, n, tot);
    note_launch();
    mf_status st = MF_OK;
    if (cudaGetLastError() != cudaSuccess) st = MF_ERR_CUDA;
    if (st == MF_OK) st = scan_rec(tot, tot, blocks, s, nullptr);
    if (st == MF_OK) {
        k_block_scan<<<blocks, SCAN_NT, 0, s>>>(in, out, n, tot, d_total);
        note_launch();
        if (cudaGetLastError() != cudaSuccess) st = MF_ERR_CUDA;
    }
    cudaFreeAsync(tot, s);
    return st;
}

}  // namespace

mf_status exclusive_scan_i32(const int *in, int *out, int n, cudaStream_t s, int *total_host)
{
    if (n <= 0) {
        if (total_host) *total_host = 0;
        return MF_OK;
    }
    int *d_total = nullptr;
    if (total_host) MF_CUDA(pool_malloc_async(&d_total, sizeof(int), s));
    mf_status st = scan_rec(in, out, n, s, d_total);
    if (total_host) {
        if (st == MF_OK) {
            cudaError_t e = cudaMemcpyAsync(total_host, d_total, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                set_last_error("scan total copy: %s", cudaGetErrorString(e));
                st = MF_ERR_CUDA;
            }
        }
        cudaFreeAsync(d_total, s);
    }
    return st;
}

}  // namespace mf
