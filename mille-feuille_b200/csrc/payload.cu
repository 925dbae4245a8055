// payload.cu -- working precision classes and the packed per-strip payload
// of the mixed-precision solver.
//
// Each tile's values are stored once per class it can be read in: FP64
// (Blockcsr_Val), FP32 (Blockcsr_Val_Low), FP16 and INT8 (built with the
// reference's casts, src/main-cg-mixed.cu:2333-2336).  A solve reads one
// packed buffer in which every tile holds its values in its current working
// class (4-byte aligned per tile), so a strip's payload stays one contiguous
// range and the bytes read per entry are those of the class.  The buffer is
// rebuilt whenever a policy changes the classes (at checkpoints).
#include <cuda_fp16.h>

#include "solver.h"

namespace mf {
namespace {

__device__ __forceinline__ int class_bytes(int c)
{
    return c == MF_CLASS_FP16 ? 2 : c == MF_CLASS_INT8 ? 1 : c == MF_CLASS_BYPASS ? 0 : 4;
}

__global__ void k_pack_sizes(int T, const int *__restrict__ tile_nnz, const unsigned char *__restrict__ wcls,
                             int *__restrict__ sizes)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += gridDim.x * blockDim.x) {
        if (t == T) {
            sizes[t] = 0;
            continue;
        }
        const int nz = tile_nnz[t + 1] - tile_nnz[t];
        sizes[t] = (nz * class_bytes(wcls[t]) + 3) & ~3;
    }
}

// One warp per tile: write the tile's entries in its working class.
__global__ void k_pack_fill(int T, const int *__restrict__ tile_nnz, const unsigned char *__restrict__ wcls,
                            const unsigned *__restrict__ poff, const float *__restrict__ low,
                            const uint16_t *__restrict__ f16, const int8_t *__restrict__ i8,
                            unsigned char *__restrict__ pay)
{
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += (gridDim.x * blockDim.x) >> 5) {
        const int a = tile_nnz[t], nz = tile_nnz[t + 1] - a;
        const int c = wcls[t];
        unsigned char *dst = pay + poff[t];
        for (int k = lane; k < nz; k += 32) {
            if (c == MF_CLASS_FP16) ((uint16_t *)dst)[k] = f16[a + k];
            else if (c == MF_CLASS_INT8) ((int8_t *)dst)[k] = i8[a + k];
            else if (c != MF_CLASS_BYPASS) ((float *)dst)[k] = low[a + k];
        }
    }
}

// Static policy: the stored (value-range) class; tiles that need FP64 run
// their inner products from the FP32 payload.  range16 (MF_POLICY_STATIC_FP16):
// an inexact tile whose nonzero values are all normal binary16 numbers
// (f16ok bit 1) runs from its FP16 payload instead.
__global__ void k_static_classes(int T, const unsigned char *__restrict__ cls, const unsigned char *__restrict__ ok16,
                                 int range16, unsigned char *__restrict__ w)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int c = cls[t];
        int v = (c == MF_CLASS_FP64) ? MF_CLASS_FP32 : c;
        if (range16 && v == MF_CLASS_FP32 && (ok16[t] & 2)) v = MF_CLASS_FP16;
        w[t] = (unsigned char)v;
    }
}

int grid_for(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

mf_status static_working_classes(mf_matrix m, unsigned char *d_wcls, cudaStream_t s, bool range16)
{
    const int T = m->v.tilenum;
    if (T == 0) return MF_OK;
    k_static_classes<<<grid_for(T, 256), 256, 0, s>>>(T, m->d_class, m->d_f16ok, range16 ? 1 : 0, d_wcls);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

mf_status pack_payload(mf_matrix m, const unsigned char *d_wcls, cudaStream_t s)
{
    const int T = m->v.tilenum;
    if (!m->d_poff) MF_CUDA(cudaMalloc(&m->d_poff, sizeof(unsigned) * (T + 1) + 16));
    int *sizes = nullptr;
    MF_CUDA(pool_malloc_async(&sizes, sizeof(int) * (T + 1), s));
    k_pack_sizes<<<grid_for(T + 1, 256), 256, 0, s>>>(T, m->d_tile_nnz, d_wcls, sizes);
    note_launch();
    MF_CUDA(cudaGetLastError());
    int total = 0;
    MF_TRY(exclusive_scan_i32(sizes, (int *)m->d_poff, T + 1, s, &total));
    cudaFreeAsync(sizes, s);
    if (total < 0) {
        set_last_error("packed payload above 2 GiB");
        return MF_ERR_UNSUPPORTED;
    }
    const size_t need = (size_t)total + 32;
    if (m->pay_bytes < need) {
        if (m->d_pay) cudaFree(m->d_pay);
        m->d_pay = nullptr;
        m->pay_bytes = 0;
        // the largest packing (every tile FP32) bounds all later ones
        const size_t cap = (size_t)m->v.nnz * 4 + (size_t)T * 4 + 32;
        MF_CUDA(cudaMalloc(&m->d_pay, cap > need ? cap : need));
        m->pay_bytes = cap > need ? cap : need;
    }
    if (T > 0) {
        k_pack_fill<<<grid_for((long long)T * 32, 256), 256, 0, s>>>(T, m->d_tile_nnz, d_wcls, m->d_poff, m->d_val_low,
                                                                    m->d_f16, m->d_i8, m->d_pay);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    m->pay_used = (size_t)total;
    return MF_OK;
}

}  // namespace mf

namespace mf {
namespace {

// max |p| per 16-column segment (as float bits: non-negative floats order
// like their bit patterns) and over the whole vector.
template <typename VT>
__global__ void k_seg_change(int nseg, int n, const VT *__restrict__ pn, const VT *__restrict__ po,
                             float *__restrict__ seg_dp, unsigned *__restrict__ pmax_bits)
{
    const int lane = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < nseg; s += (gridDim.x * blockDim.x) >> 4) {
        const int j = s * MF_TILE + lane;
        float dp = 0.f, pm = 0.f;
        if (j < n) {
            dp = fabsf((float)pn[j] - (float)po[j]);
            pm = fabsf((float)pn[j]);
        }
        for (int o = 8; o > 0; o >>= 1) {
            dp = fmaxf(dp, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), dp, o, 16));
            pm = fmaxf(pm, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), pm, o, 16));
        }
        if (lane == 0) {
            seg_dp[s] = dp;
            atomicMax(pmax_bits, __float_as_uint(pm));
        }
    }
}

// The reference's partial-convergence decision (src/main-cg-mixed.cu:415-460)
// per 16-row segment of p, after the p update: v = |p_new - p_old| of every
// element, in FP64;  v > 1e-5 -> FP64, 1e-6 < v <= 1e-5 -> FP32,
// 1e-7 < v <= 1e-6 -> FP16, 1e-8 < v <= 1e-7 -> INT8, else BYPASS.  The
// reference's lanes race on one shared word; here the most precise class any
// element of the segment demands wins (the class of the largest v).
template <typename VT>
__global__ void k_seg_rule(int nseg, int n, const VT *__restrict__ pn, const VT *__restrict__ po,
                           unsigned char *__restrict__ seg_cls)
{
    const int lane = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < nseg; s += (gridDim.x * blockDim.x) >> 4) {
        const int j = s * MF_TILE + lane;
        double v = 0.0;
        if (j < n) v = fabs((double)pn[j] - (double)po[j]);
        for (int o = 8; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), v, o, 16));
        if (lane == 0) {
            int c;
            if (v > 1e-5) c = MF_CLASS_FP64;
            else if (v > 1e-6) c = MF_CLASS_FP32;
            else if (v > 1e-7) c = MF_CLASS_FP16;
            else if (v > 1e-8) c = MF_CLASS_INT8;
            else c = MF_CLASS_BYPASS;
            seg_cls[s] = (unsigned char)c;
        }
    }
}

// The class the mixed solver executes a tile in, for a decided class d and
// the tile's exact (value-range) class c: the FP32 payload for FP64 / FP32
// decisions (the inner solver's vectors and sums are FP32; FP64 accuracy
// comes from the reliable updates), FP16 for FP16 and for INT8 decisions on
// tiles that are not integers, and an exact class narrower than the decided
// one is kept.  A BYPASS decision drops the tile only under the scaled rule
// (keep_bypass): the absolute thresholds call every segment converged once
// |p| itself falls below 1e-8, which would empty the product, so there it
// runs like an INT8 decision.  An inexact tile whose FP16 payload is not
// finite (ok16 = 0) runs FP16 decisions in FP32.
__device__ __forceinline__ int exec_class(int d, int c, bool keep_bypass, bool ok16)
{
    int w;
    if (d == MF_CLASS_FP64 || d == MF_CLASS_FP32) w = MF_CLASS_FP32;
    else if (d == MF_CLASS_FP16) w = MF_CLASS_FP16;
    else if (d == MF_CLASS_INT8 || !keep_bypass) w = (c == MF_CLASS_INT8) ? MF_CLASS_INT8 : MF_CLASS_FP16;
    else w = MF_CLASS_BYPASS;
    if (w == MF_CLASS_FP32 && (c == MF_CLASS_FP16 || c == MF_CLASS_INT8)) w = c;
    if (w == MF_CLASS_FP16 && c == MF_CLASS_INT8) w = c;
    if (w == MF_CLASS_FP16 && c != MF_CLASS_FP16 && !ok16) w = MF_CLASS_FP32;
    return w;
}

// Tile t takes the decision of its column segment (the p segment it
// multiplies), as the reference's SpMV reads d_vis[tile column].
__global__ void k_rule_tiles(int T, const int *__restrict__ tile_col, const unsigned char *__restrict__ cls,
                             const unsigned char *__restrict__ ok16, const unsigned char *__restrict__ seg_cls,
                             unsigned char *__restrict__ decision,
                             unsigned char *__restrict__ w)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int d = seg_cls[tile_col[t]];
        if (decision) decision[t] = (unsigned char)d;
        if (w) w[t] = (unsigned char)exec_class(d, cls[t], false, (ok16[t] & 1) != 0);
    }
}

// MF_POLICY_RULE_SCALED: the same thresholds on the change relative to the
// largest |p| (float), so that the decision does not depend on the scale of
// b: v = max_seg |p_new - p_old| / max |p_new|;  v > 1e-6 -> FP32,
// 1e-7 < v <= 1e-6 -> FP16, 1e-8 < v <= 1e-7 -> INT8, else BYPASS (no FP64
// decision: FP32 is the inner solver's widest class).
__global__ void k_rule_scaled_classes(int T, const int *__restrict__ tile_col, const unsigned char *__restrict__ cls,
                                      const unsigned char *__restrict__ ok16, const float *__restrict__ seg_dp, const unsigned *__restrict__ pmax_bits,
                                      unsigned char *__restrict__ decision, unsigned char *__restrict__ w)
{
    const float pmax = __uint_as_float(*pmax_bits);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const float v = pmax > 0.f ? seg_dp[tile_col[t]] / pmax : 0.f;
        int d;
        if (v > 1e-6f) d = MF_CLASS_FP32;
        else if (v > 1e-7f) d = MF_CLASS_FP16;
        else if (v > 1e-8f) d = MF_CLASS_INT8;
        else d = MF_CLASS_BYPASS;
        if (decision) decision[t] = (unsigned char)d;
        if (w) w[t] = (unsigned char)exec_class(d, cls[t], true, (ok16[t] & 1) != 0);
    }
}

int grid_for2(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

mf_status rule_classes(mf_matrix m, int policy, const void *p_new, const void *p_old, unsigned char *d_decision,
                       unsigned char *d_wcls, cudaStream_t s)
{
    const int T = m->v.tilenum, n = m->v.cols;
    const int nseg = m->v.tilen;
    if (policy == MF_POLICY_RULE) {
        unsigned char *seg = nullptr;
        MF_CUDA(pool_malloc_async(&seg, (size_t)nseg + 16, s));
        if (nseg > 0) {
            k_seg_rule<float><<<grid_for2((long long)nseg * 16, 256), 256, 0, s>>>(nseg, n, (const float *)p_new,
                                                                                  (const float *)p_old, seg);
            note_launch();
            MF_CUDA(cudaGetLastError());
        }
        if (T > 0) {
            k_rule_tiles<<<grid_for2(T, 256), 256, 0, s>>>(T, m->d_tile_columnidx, m->d_class, m->d_f16ok, seg, d_decision,
                                                              d_wcls);
            note_launch();
            MF_CUDA(cudaGetLastError());
        }
        cudaFreeAsync(seg, s);
        return MF_OK;
    }
    float *seg = nullptr;
    MF_CUDA(pool_malloc_async(&seg, sizeof(float) * nseg + sizeof(unsigned) * 4, s));
    unsigned *pmax = (unsigned *)(seg + nseg);
    MF_CUDA(cudaMemsetAsync(pmax, 0, sizeof(unsigned), s));
    if (nseg > 0) {
        k_seg_change<float><<<grid_for2((long long)nseg * 16, 256), 256, 0, s>>>(nseg, n, (const float *)p_new,
                                                                                 (const float *)p_old, seg, pmax);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    if (T > 0) {
        k_rule_scaled_classes<<<grid_for2(T, 256), 256, 0, s>>>(T, m->d_tile_columnidx, m->d_class, m->d_f16ok, seg, pmax,
                                                                 d_decision, d_wcls);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    cudaFreeAsync(seg, s);
    return MF_OK;
}

}  // namespace mf

extern "C" mf_status mf_rule_classes(mf_matrix m, int policy, const float *p_new, const float *p_old,
                                     unsigned char *decision, unsigned char *working, void *stream)
{
    if (!m || (policy != MF_POLICY_RULE && policy != MF_POLICY_RULE_SCALED) ||
        (m->v.cols > 0 && (!p_new || !p_old))) {
        mf::set_last_error("mf_rule_classes: null argument or policy other than RULE / RULE_SCALED");
        return MF_ERR_INVALID_ARG;
    }
    return mf::rule_classes(m, policy, p_new, p_old, decision, working, (cudaStream_t)stream);
}
