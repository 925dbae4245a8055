// policy.cu -- the learned per-tile precision policy.
//
// No reference counterpart: the reference picks a class per 16-row segment
// from how much p changed (src/main-cg-mixed.cu:415-460).  Here a small MLP
// (16 features -> 32 -> 32 -> 4 classes, BF16 weights, FP32 accumulation)
// predicts each tile's class at every checkpoint of a mixed solve.
//
// Features of tile t (row strip i, column segment j), all from device data:
//   0 log10 max|a| / 10        1 log10 min|a| / 10     2 entries / 256
//   3 diagonal tile            4 integer tile (int8)   5 fp16-exact tile
//   6 log10(max_j|p| / max|p|)/10     7 log10(max_j|p - p_old| / max|p|)/10
//   8 log10(max_i|r| / max|r|)/10     9 log10(||r|| / ||b||)/10
//  10 log10(max|a| max_j|p| / max|q|)/10
//  11..14 features 6, 7, 8, 9 at the previous checkpoint (history)
//  15 1 (bias input)
// Labels (from FP64 solver traces): the narrowest class whose rounding costs
// no more than the FP32 rounding of the rows the tile feeds (k_collect):
//   0 int8 (exact integer tile) or bypass, 1 fp16, 2 fp32 (3 fp64: unused).
// Training: softmax cross-entropy, per-sample backward in shared memory,
// per-parameter sums over the samples in a fixed order (deterministic), Adam
// on FP32 master weights, BF16 copies for the forward pass.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "policy_net.cuh"
#include "solver.h"

namespace mf {
constexpr int NF = PN_NF, H1 = PN_H1, H2 = PN_H2, NO = PN_NO;
constexpr int OW1 = PN_OW1, OB1 = PN_OB1, OW2 = PN_OW2, OB2 = PN_OB2, OW3 = PN_OW3, OB3 = PN_OB3;
constexpr int NPARAM = PN_NPARAM;  // 1732
}  // namespace mf

struct mf_policy_s {
    float *d_master = nullptr, *d_m = nullptr, *d_v = nullptr;  // FP32 master weights, Adam moments
    __nv_bfloat16 *d_w = nullptr;                                 // BF16 weights (forward pass)
    long long steps = 0;
    // training samples
    float *d_x = nullptr;
    unsigned char *d_y = nullptr;
    long long n = 0, cap = 0;
    long long label_counts[4] = {0, 0, 0, 0};
};

namespace mf {
namespace {

__device__ __forceinline__ float safe_log10(float v) { return log10f(fmaxf(v, 1e-30f)); }

// ---- segment statistics and features ------------------------------------

template <typename VT>
__global__ void k_seg_stats(int nseg, int n, const VT *__restrict__ pn, const VT *__restrict__ po,
                            const VT *__restrict__ r, float *__restrict__ sp, float *__restrict__ sdp,
                            float *__restrict__ sr, unsigned *__restrict__ gmax /*[0] p, [1] r*/)
{
    const int lane = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < nseg; s += (gridDim.x * blockDim.x) >> 4) {
        const int j = s * MF_TILE + lane;
        float p = 0.f, dp = 0.f, rr = 0.f;
        if (j < n) {
            p = fabsf((float)pn[j]);
            dp = fabsf((float)pn[j] - (float)po[j]);
            rr = fabsf((float)r[j]);
        }
        for (int o = 8; o > 0; o >>= 1) {
            p = fmaxf(p, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), p, o, 16));
            dp = fmaxf(dp, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), dp, o, 16));
            rr = fmaxf(rr, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), rr, o, 16));
        }
        if (lane == 0) {
            sp[s] = p;
            sdp[s] = dp;
            sr[s] = rr;
            atomicMax(&gmax[0], __float_as_uint(p));
            atomicMax(&gmax[1], __float_as_uint(rr));
        }
    }
}

// per-tile static features: max |a|, min |a| (nonzero), entries; kept on the
// policy workspace of the matrix
__global__ void k_tile_static(int T, const int *__restrict__ tile_nnz, const double *__restrict__ val,
                              float *__restrict__ vmax, float *__restrict__ vmin)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        float mx = 0.f, mn = 3.0e38f;
        for (int k = tile_nnz[t]; k < tile_nnz[t + 1]; k++) {
            const float a = (float)fabs(val[k]);
            mx = fmaxf(mx, a);
            if (a > 0.f) mn = fminf(mn, a);
        }
        vmax[t] = mx;
        vmin[t] = (mn > 1e38f) ? 0.f : mn;
    }
}

struct FeatIn {
    int T;
    const int *tile_col, *tile_row, *tile_nnz;
    const unsigned char *cls;
    const float *vmax, *vmin;
    const float *sp, *sdp, *sr;             // current segment stats
    const float *psp, *psdp, *psr;          // previous checkpoint
    const unsigned *gmax;                   // [0] max|p|, [1] max|r|, [2] max|q| (bits)
    float relres, prev_relres;
};

__device__ __forceinline__ void tile_features(const FeatIn &f, int t, float *x)
{
    const int j = f.tile_col[t], i = f.tile_row[t];
    const float pmax = __uint_as_float(f.gmax[0]), rmax = __uint_as_float(f.gmax[1]);
    const float qmax = __uint_as_float(f.gmax[2]);
    const float inv_p = pmax > 0.f ? 1.f / pmax : 0.f, inv_r = rmax > 0.f ? 1.f / rmax : 0.f;
    x[0] = safe_log10(f.vmax[t]) * 0.1f;
    x[1] = safe_log10(f.vmin[t]) * 0.1f;
    x[2] = (float)(f.tile_nnz[t + 1] - f.tile_nnz[t]) * (1.f / 256.f);
    x[3] = (i == j) ? 1.f : 0.f;
    x[4] = (f.cls[t] == MF_CLASS_INT8) ? 1.f : 0.f;
    x[5] = (f.cls[t] == MF_CLASS_FP16) ? 1.f : 0.f;
    x[6] = safe_log10(f.sp[j] * inv_p) * 0.1f;
    x[7] = safe_log10(f.sdp[j] * inv_p) * 0.1f;
    x[8] = safe_log10(f.sr[i] * inv_r) * 0.1f;
    x[9] = safe_log10(f.relres) * 0.1f;
    x[10] = safe_log10(f.vmax[t] * f.sp[j] / fmaxf(qmax, 1e-30f)) * 0.1f;
    x[11] = f.psp ? safe_log10(f.psp[j] * inv_p) * 0.1f : x[6];
    x[12] = f.psdp ? safe_log10(f.psdp[j] * inv_p) * 0.1f : x[7];
    x[13] = f.psr ? safe_log10(f.psr[i] * inv_r) * 0.1f : x[8];
    x[14] = f.prev_relres > 0.f ? safe_log10(f.prev_relres) * 0.1f : x[9];
    x[15] = 1.f;
}

// |A| |p| per row (the magnitude the row's FP32 sum is rounded against).
__global__ void k_row_absmag(MfTiles A, const double *__restrict__ p, double *__restrict__ mag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.rows; i += gridDim.x * blockDim.x) {
        const int bi = i / MF_TILE, r = i % MF_TILE;
        const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
        double m = 0.0;
        for (int t = A.tile_ptr[bi]; t < A.tile_ptr[bi + 1]; t++) {
            const int off = A.tile_nnz[t], nz = A.tile_nnz[t + 1] - off;
            const int po = A.csrptr_offset[t];
            const int lo = A.ptr[po + r], hi = (r == rowlen - 1) ? nz : (int)A.ptr[po + r + 1];
            const int xo = A.tile_columnidx[t] * MF_TILE;
            for (int k = lo; k < hi; k++) m += fabs(A.val[off + k]) * fabs(p[xo + A.col[off + k]]);
        }
        mag[i] = m;
    }
}

// Label of a tile: the narrowest class whose rounding costs no more than the
// FP32 rounding of the rows it feeds.  With e_r = sum |a||p| over the tile's
// entries of row r and M_r the same sum over the whole row, storing the tile
// in fp16 adds about 2^-11 e_r and skipping it adds e_r, against the FP32
// sum's 2^-24 M_r:  0 (int8-exact tile, or every e_r <= 2^-24 M_r: bypass),
// 1 (fp16-exact tile, or every e_r <= 2^-13 M_r), 2 (fp32).  Class 3 (fp64)
// is never needed by the inner FP32 solver.
template <typename VT>
__global__ void k_collect(FeatIn f, const double *__restrict__ val, const unsigned char *__restrict__ col,
                          const unsigned char *__restrict__ ptr, int last_tile_begin, int last_rowlen,
                          const VT *__restrict__ pn, const double *__restrict__ mag, int stride, unsigned salt,
                          float *__restrict__ X, unsigned char *__restrict__ Y, unsigned long long *__restrict__ count,
                          long long cap)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < f.T; t += gridDim.x * blockDim.x) {
        const unsigned h = (unsigned)t * 2654435761u ^ salt;
        if ((h >> 8) % (unsigned)stride != 0u) continue;
        const int o0 = f.tile_nnz[t], nz = f.tile_nnz[t + 1] - o0;
        const long long po = (t < last_tile_begin) ? 16ll * t : 16ll * last_tile_begin + (long long)(t - last_tile_begin) * last_rowlen;
        const int rowlen = (t < last_tile_begin) ? MF_TILE : last_rowlen;
        const int xo = f.tile_col[t] * MF_TILE;
        const int row0 = f.tile_row[t] * MF_TILE;
        double ratio = 0.0;  // max_r e_r / M_r
        for (int r = 0; r < rowlen; r++) {
            const int lo = ptr[po + r], hi = (r == rowlen - 1) ? nz : (int)ptr[po + r + 1];
            double e = 0.0;
            for (int k = lo; k < hi; k++) e += fabs(val[o0 + k]) * fabs((double)pn[xo + col[o0 + k]]);
            const double M = mag[row0 + r];
            if (e > 0.0) ratio = fmax(ratio, M > 0.0 ? e / M : 1.0);
        }
        int lab;
        if (f.cls[t] == MF_CLASS_INT8 || ratio <= 0x1.0p-24) lab = 0;
        else if (f.cls[t] == MF_CLASS_FP16 || ratio <= 0x1.0p-13) lab = 1;
        else lab = 2;
        const unsigned long long slot = atomicAdd(count, 1ull);
        if ((long long)slot >= cap) continue;
        float x[NF];
        tile_features(f, t, x);
        for (int k = 0; k < NF; k++) X[slot * NF + k] = x[k];
        Y[slot] = (unsigned char)lab;
    }
}

__global__ void k_absmax(long long n, const void *q, int is_float, unsigned *out)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(is_float ? ((const float *)q)[i] : (float)((const double *)q)[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// ---- MLP -------------------------------------------------------------

__device__ __forceinline__ void load_weights(const __nv_bfloat16 *__restrict__ w, float *s_w)
{
    for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) s_w[k] = __bfloat162float(w[k]);
    __syncthreads();
}

__device__ __forceinline__ void mlp_forward(const float *w, const float *x, float *h1, float *h2, float *out)
{
    pn_forward(w, x, h1, h2, out);
}

__global__ void k_mlp_classify(FeatIn f, const __nv_bfloat16 *__restrict__ wq, unsigned char *__restrict__ wcls)
{
    __shared__ float s_w[NPARAM];
    load_weights(wq, s_w);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < f.T; t += gridDim.x * blockDim.x) {
        float x[NF], h1[H1], h2[H2], o[NO];
        tile_features(f, t, x);
        mlp_forward(s_w, x, h1, h2, o);
        // conservative decision: the narrowest class c the network is 99 %
        // sure the tile tolerates, P(label <= c) >= 0.99
        float mx = o[0];
        for (int k = 1; k < NO; k++) mx = fmaxf(mx, o[k]);
        float pr[NO], z = 0.f;
        for (int k = 0; k < NO; k++) {
            pr[k] = __expf(o[k] - mx);
            z += pr[k];
        }
        int best = NO - 1;
        float cum = 0.f;
        for (int k = 0; k < NO; k++) {
            cum += pr[k];
            if (cum >= 0.99f * z) {
                best = k;
                break;
            }
        }
        const int c = f.cls[t];
        int w;
        if (best == 0) w = (c == MF_CLASS_INT8) ? MF_CLASS_INT8 : MF_CLASS_BYPASS;
        else if (best == 1) w = (c == MF_CLASS_INT8) ? MF_CLASS_INT8 : MF_CLASS_FP16;
        else w = (c == MF_CLASS_INT8 || c == MF_CLASS_FP16) ? c : MF_CLASS_FP32;
        // an inexact tile beyond binary16's range stays FP32
        if (w == MF_CLASS_FP16 && c != MF_CLASS_FP16 && !(f.vmax[t] <= 65504.f)) w = MF_CLASS_FP32;
        wcls[t] = (unsigned char)w;
    }
}

constexpr int TB = 128;  // samples per training block
constexpr int SROW = NF + H1 + H2 + NO + H2 + H1;  // per-sample activations and deltas

// Forward + backward of TB samples; writes this block's gradient sums (in a
// fixed sample order) and loss sum.  grad of the mean loss when scaled by 1/B.
__global__ void __launch_bounds__(TB) k_mlp_grad(const __nv_bfloat16 *__restrict__ wq, const float *__restrict__ X,
                                                 const unsigned char *__restrict__ Y, const long long *__restrict__ idx,
                                                 long long i0, int B, float scale, float *__restrict__ gpart,
                                                 float *__restrict__ lpart)
{
    extern __shared__ float sm[];
    float *s_w = sm;
    float *s_a = sm + NPARAM + 4;
    for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) s_w[k] = __bfloat162float(wq[k]);
    __syncthreads();
    const int sidx = blockIdx.x * TB + threadIdx.x;
    float *a = s_a + threadIdx.x * SROW;
    float *x = a, *h1 = a + NF, *h2 = h1 + H1, *dl = h2 + H2, *d2 = dl + NO, *d1 = d2 + H2;
    float loss = 0.f;
    if (sidx < B) {
        const long long si = idx ? idx[i0 + sidx] : i0 + sidx;
        for (int k = 0; k < NF; k++) x[k] = X[si * NF + k];
        float o[NO];
        mlp_forward(s_w, x, h1, h2, o);
        float mx = o[0];
        for (int k = 1; k < NO; k++) mx = fmaxf(mx, o[k]);
        float z = 0.f;
        for (int k = 0; k < NO; k++) z += expf(o[k] - mx);
        const int y = Y[si];
        loss = -(o[y] - mx - logf(z));
        for (int k = 0; k < NO; k++) dl[k] = (expf(o[k] - mx) / z - (k == y ? 1.f : 0.f)) * scale;
        for (int j = 0; j < H2; j++) {
            float s = 0.f;
            for (int k = 0; k < NO; k++) s = fmaf(s_w[OW3 + k * H2 + j], dl[k], s);
            d2[j] = h2[j] > 0.f ? s : 0.f;
        }
        for (int j = 0; j < H1; j++) {
            float s = 0.f;
            for (int k = 0; k < H2; k++) s = fmaf(s_w[OW2 + k * H1 + j], d2[k], s);
            d1[j] = h1[j] > 0.f ? s : 0.f;
        }
    } else {
        for (int k = 0; k < SROW; k++) a[k] = 0.f;
    }
    __syncthreads();
    const int ns = min(TB, B - blockIdx.x * TB);
    for (int p = threadIdx.x; p < NPARAM; p += blockDim.x) {
        float g = 0.f;
        for (int s = 0; s < ns; s++) {
            const float *as = s_a + s * SROW;
            const float *sx = as, *sh1 = as + NF, *sh2 = sh1 + H1, *sdl = sh2 + H2, *sd2 = sdl + NO, *sd1 = sd2 + H2;
            if (p < OB1) g = fmaf(sd1[p / NF], sx[p % NF], g);
            else if (p < OW2) g += sd1[p - OB1];
            else if (p < OB2) g = fmaf(sd2[(p - OW2) / H1], sh1[(p - OW2) % H1], g);
            else if (p < OW3) g += sd2[p - OB2];
            else if (p < OB3) g = fmaf(sdl[(p - OW3) / H2], sh2[(p - OW3) % H2], g);
            else g += sdl[p - OB3];
        }
        gpart[(size_t)blockIdx.x * NPARAM + p] = g;
    }
    // loss: fixed tree
    __shared__ float s_l[TB];
    s_l[threadIdx.x] = loss;
    __syncthreads();
    for (int o = TB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s_l[threadIdx.x] += s_l[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) lpart[blockIdx.x] = s_l[0];
}

// Sum the block gradients in block order; Adam step when lr > 0; BF16 copy.
__global__ void k_mlp_update(int nblk, const float *__restrict__ gpart, float *__restrict__ grad_out,
                             float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                             __nv_bfloat16 *__restrict__ wq, float lr, long long step)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NPARAM; p += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (int b = 0; b < nblk; b++) g += gpart[(size_t)b * NPARAM + p];
        if (grad_out) grad_out[p] = g;
        if (lr > 0.f) {
            const float b1 = 0.9f, b2 = 0.999f;
            m[p] = b1 * m[p] + (1.f - b1) * g;
            v[p] = b2 * v[p] + (1.f - b2) * g * g;
            const float mh = m[p] / (1.f - powf(b1, (float)step)), vh = v[p] / (1.f - powf(b2, (float)step));
            w[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
            wq[p] = __float2bfloat16_rn(w[p]);
        }
    }
}

int grid_for4(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

// Per-matrix policy workspace: static tile features, tile row index,
// segment statistics of the current and previous checkpoint.
struct PolicyWork {
    float *vmax, *vmin, *sp, *sdp, *sr, *psp, *psdp, *psr;
    unsigned *gmax;
    float prev_relres;
    int have_prev;
    int ns;  // segment slots per statistic (max of tile rows and tile columns)
};

static mf_status policy_work(mf_matrix m, PolicyWork &pw, cudaStream_t s)
{
    const int T = m->v.tilenum, ns = m->v.tilen > m->v.tilem ? m->v.tilen : m->v.tilem;
    const size_t need = sizeof(float) * ((size_t)2 * T + 6 * (size_t)ns + 64) + 64;
    if (m->pol_bytes < need) {
        if (m->d_pol) cudaFree(m->d_pol);
        m->d_pol = nullptr;
        m->pol_bytes = 0;
        MF_CUDA(cudaMalloc(&m->d_pol, need));
        m->pol_bytes = need;
        m->pol_static_ready = 0;
        m->pol_have_prev = 0;
    }
    float *b = (float *)m->d_pol;
    pw.vmax = b;
    pw.vmin = b + T;
    pw.sp = b + 2 * (size_t)T;
    pw.sdp = pw.sp + ns;
    pw.sr = pw.sdp + ns;
    pw.psp = pw.sr + ns;
    pw.psdp = pw.psp + ns;
    pw.psr = pw.psdp + ns;
    pw.gmax = (unsigned *)(pw.psr + ns);
    pw.ns = ns;
    if (!m->pol_static_ready && T > 0) {
        k_tile_static<<<grid_for4(T, 256), 256, 0, s>>>(T, m->d_tile_nnz, m->d_val, pw.vmax, pw.vmin);
        note_launch();
        MF_CUDA(cudaGetLastError());
        m->pol_static_ready = 1;
    }
    pw.prev_relres = m->pol_prev_relres;
    pw.have_prev = m->pol_have_prev;
    return MF_OK;
}

// Segment statistics of the current checkpoint; previous ones rotate.
template <typename VT>
static mf_status checkpoint_stats(mf_matrix m, PolicyWork &pw, const void *pnew, const void *pold, const void *r,
                                  const void *q, cudaStream_t s)
{
    const int ns = m->v.tilen, n = m->v.cols;
    if (pw.have_prev) {
        MF_CUDA(cudaMemcpyAsync(pw.psp, pw.sp, sizeof(float) * (size_t)pw.ns * 3, cudaMemcpyDeviceToDevice, s));
    }
    MF_CUDA(cudaMemsetAsync(pw.gmax, 0, sizeof(unsigned) * 4, s));
    k_seg_stats<VT><<<grid_for4((long long)ns * 16, 256), 256, 0, s>>>(ns, n, (const VT *)pnew, (const VT *)pold,
                                                                       (const VT *)r, pw.sp, pw.sdp, pw.sr, pw.gmax);
    note_launch();
    MF_CUDA(cudaGetLastError());
    k_absmax<<<grid_for4(n, 256), 256, 0, s>>>(n, q, sizeof(VT) == 4 ? 1 : 0, pw.gmax + 2);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

static FeatIn feat_in(mf_matrix m, const PolicyWork &pw, float relres)
{
    FeatIn f;
    f.T = m->v.tilenum;
    f.tile_col = m->d_tile_columnidx;
    f.tile_row = m->d_tile_rowidx;
    f.tile_nnz = m->d_tile_nnz;
    f.cls = m->d_class;
    f.vmax = pw.vmax;
    f.vmin = pw.vmin;
    f.sp = pw.sp;
    f.sdp = pw.sdp;
    f.sr = pw.sr;
    f.psp = pw.have_prev ? pw.psp : nullptr;
    f.psdp = pw.have_prev ? pw.psdp : nullptr;
    f.psr = pw.have_prev ? pw.psr : nullptr;
    f.gmax = pw.gmax;
    f.relres = relres;
    f.prev_relres = pw.have_prev ? pw.prev_relres : 0.f;
    return f;
}

mf_status learned_working_classes(mf_matrix m, SolverWork &w, const void *p_new, const void *p_old,
                                  unsigned char *d_wcls, cudaStream_t s)
{
    mf_learned p = m->policy;
    if (!p) {
        set_last_error("learned policy not attached");
        return MF_ERR_UNSUPPORTED;
    }
    PolicyWork pw;
    MF_TRY(policy_work(m, pw, s));
    MF_TRY(checkpoint_stats<float>(m, pw, p_new, p_old, w.r, w.q, s));
    double st[S_COUNT];
    MF_CUDA(cudaMemcpyAsync(st, w.state, sizeof(st), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    const float relres = (float)st[S_RELRES];
    const FeatIn f = feat_in(m, pw, relres);
    if (f.T > 0) {
        k_mlp_classify<<<grid_for4(f.T, 256), 256, 0, s>>>(f, p->d_w, d_wcls);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    m->pol_prev_relres = relres;
    m->pol_have_prev = 1;
    return MF_OK;
}

void policy_reset_history(mf_matrix m) { m->pol_have_prev = 0; }

struct CollectCtx {
    mf_learned p;
    int stride;
    unsigned salt;
};

static mf_status collect_hook(void *ctx, mf_matrix m, SolverWork &w, const void *p_new, const void *p_old, int it,
                              double relres, cudaStream_t s)
{
    CollectCtx *c = (CollectCtx *)ctx;
    mf_learned p = c->p;
    PolicyWork pw;
    MF_TRY(policy_work(m, pw, s));
    MF_TRY(checkpoint_stats<double>(m, pw, p_new, p_old, w.r, w.q, s));
    const FeatIn f = feat_in(m, pw, (float)relres);
    unsigned long long *d_cnt = nullptr;
    MF_CUDA(pool_malloc_async(&d_cnt, sizeof(unsigned long long) + sizeof(double) * ((size_t)m->v.rows + 1), s));
    double *d_mag = (double *)(d_cnt + 1);
    if (m->v.rows > 0) {
        k_row_absmag<<<grid_for4(m->v.rows, 256), 256, 0, s>>>(m->v, (const double *)p_new, d_mag);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    const unsigned long long start = (unsigned long long)p->n;
    MF_CUDA(cudaMemcpyAsync(d_cnt, &start, sizeof(start), cudaMemcpyHostToDevice, s));
    if (f.T > 0) {
        k_collect<double><<<grid_for4(f.T, 256), 256, 0, s>>>(
            f, m->d_val, m->d_col, m->d_ptr, m->last_tile_begin, m->v.rows - (m->v.tilem - 1) * MF_TILE,
            (const double *)p_new, d_mag, c->stride, c->salt ^ (unsigned)it * 0x9E3779B9u, p->d_x, p->d_y, d_cnt,
            p->cap);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    unsigned long long end = 0;
    MF_CUDA(cudaMemcpyAsync(&end, d_cnt, sizeof(end), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(d_cnt, s);
    p->n = (long long)std::min<unsigned long long>(end, (unsigned long long)p->cap);
    m->pol_prev_relres = (float)relres;
    m->pol_have_prev = 1;
    return MF_OK;
}

}  // namespace mf

using namespace mf;

// Sample storage of the training set for the batched solver's collector:
// grows the buffers to max_samples (keeping the samples held) and returns
// them with the current sample count.
namespace mf {
mf_status policy_sample_buffers(mf_learned p, long long max_samples, float **x, unsigned char **y, long long *n)
{
    if (max_samples > p->cap) {
        float *nx = nullptr;
        unsigned char *ny = nullptr;
        MF_CUDA(cudaMalloc(&nx, sizeof(float) * NF * (size_t)max_samples));
        MF_CUDA(cudaMalloc(&ny, (size_t)max_samples + 16));
        if (p->n) {
            MF_CUDA(cudaMemcpy(nx, p->d_x, sizeof(float) * NF * (size_t)p->n, cudaMemcpyDeviceToDevice));
            MF_CUDA(cudaMemcpy(ny, p->d_y, (size_t)p->n, cudaMemcpyDeviceToDevice));
        }
        if (p->d_x) cudaFree(p->d_x);
        if (p->d_y) cudaFree(p->d_y);
        p->d_x = nx;
        p->d_y = ny;
        p->cap = max_samples;
    }
    *x = p->d_x;
    *y = p->d_y;
    *n = p->n;
    return MF_OK;
}

mf_status policy_sample_commit(mf_learned p, long long n_total)
{
    p->n = std::min(n_total, p->cap);
    return MF_OK;
}

const __nv_bfloat16 *policy_weights(mf_learned p) { return p->d_w; }
}  // namespace mf

extern "C" {

mf_status mf_policy_create(uint64_t seed, mf_learned *out)
{
    if (!out) return MF_ERR_INVALID_ARG;
    mf_learned p = new mf_policy_s();
    std::vector<float> w(NPARAM, 0.f);
    // He-style uniform init from the seed
    auto u = [&](uint64_t i) { return (double)(mix64(seed * 0x9E3779B97F4A7C15ull + i + 1) >> 11) * 0x1.0p-53; };
    for (int k = 0; k < H1 * NF; k++) w[OW1 + k] = (float)((2 * u(k) - 1) * sqrt(6.0 / NF));
    for (int k = 0; k < H2 * H1; k++) w[OW2 + k] = (float)((2 * u(10000 + k) - 1) * sqrt(6.0 / H1));
    for (int k = 0; k < NO * H2; k++) w[OW3 + k] = (float)((2 * u(20000 + k) - 1) * sqrt(6.0 / H2));
    std::vector<__nv_bfloat16> wq(NPARAM);
    for (int k = 0; k < NPARAM; k++) wq[k] = __float2bfloat16_rn(w[k]);
    cudaError_t e = cudaMalloc(&p->d_master, sizeof(float) * NPARAM * 3);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_w, sizeof(__nv_bfloat16) * NPARAM);
    if (e != cudaSuccess) {
        mf_policy_destroy(p);
        set_last_error("mf_policy_create: %s", cudaGetErrorString(e));
        return MF_ERR_NO_MEMORY;
    }
    p->d_m = p->d_master + NPARAM;
    p->d_v = p->d_master + 2 * NPARAM;
    cudaMemcpy(p->d_master, w.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice);
    cudaMemset(p->d_m, 0, sizeof(float) * NPARAM * 2);
    cudaMemcpy(p->d_w, wq.data(), sizeof(__nv_bfloat16) * NPARAM, cudaMemcpyHostToDevice);
    *out = p;
    return MF_OK;
}

mf_status mf_policy_destroy(mf_learned p)
{
    if (!p) return MF_OK;
    if (p->d_master) cudaFree(p->d_master);
    if (p->d_w) cudaFree(p->d_w);
    if (p->d_x) cudaFree(p->d_x);
    if (p->d_y) cudaFree(p->d_y);
    delete p;
    return MF_OK;
}

int mf_policy_param_count(void) { return NPARAM; }

// BF16 weights (as float) in the layout W1[32][16], b1[32], W2[32][32],
// b2[32], W3[4][32], b3[4].
mf_status mf_policy_get_params(mf_learned p, float *host, int count)
{
    if (!p || !host || count != NPARAM) return MF_ERR_INVALID_ARG;
    std::vector<__nv_bfloat16> wq(NPARAM);
    MF_CUDA(cudaMemcpy(wq.data(), p->d_w, sizeof(__nv_bfloat16) * NPARAM, cudaMemcpyDeviceToHost));
    for (int k = 0; k < NPARAM; k++) host[k] = __bfloat162float(wq[k]);
    return MF_OK;
}

mf_status mf_policy_set_params(mf_learned p, const float *host, int count)
{
    if (!p || !host || count != NPARAM) return MF_ERR_INVALID_ARG;
    std::vector<__nv_bfloat16> wq(NPARAM);
    for (int k = 0; k < NPARAM; k++) wq[k] = __float2bfloat16_rn(host[k]);
    MF_CUDA(cudaMemcpy(p->d_master, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
    MF_CUDA(cudaMemset(p->d_m, 0, sizeof(float) * NPARAM * 2));
    MF_CUDA(cudaMemcpy(p->d_w, wq.data(), sizeof(__nv_bfloat16) * NPARAM, cudaMemcpyHostToDevice));
    p->steps = 0;
    return MF_OK;
}

mf_status mf_policy_save(mf_learned p, const char *path)
{
    if (!p || !path) return MF_ERR_INVALID_ARG;
    std::vector<float> w(NPARAM);
    MF_CUDA(cudaMemcpy(w.data(), p->d_master, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_last_error("cannot write %s", path);
        return MF_ERR_IO;
    }
    const char magic[8] = {'M', 'F', 'P', 'O', 'L', '1', 0, 0};
    const int np = NPARAM;
    bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(&np, sizeof(int), 1, f) == 1 &&
              fwrite(w.data(), sizeof(float), NPARAM, f) == (size_t)NPARAM;
    fclose(f);
    return ok ? MF_OK : MF_ERR_IO;
}

mf_status mf_policy_load(const char *path, mf_learned *out)
{
    if (!path || !out) return MF_ERR_INVALID_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_last_error("cannot read %s", path);
        return MF_ERR_IO;
    }
    char magic[8];
    int np = 0;
    std::vector<float> w(NPARAM);
    bool ok = fread(magic, 1, 8, f) == 8 && !memcmp(magic, "MFPOL1", 6) && fread(&np, sizeof(int), 1, f) == 1 &&
              np == NPARAM && fread(w.data(), sizeof(float), NPARAM, f) == (size_t)NPARAM;
    fclose(f);
    if (!ok) {
        set_last_error("%s is not a policy file of this build", path);
        return MF_ERR_IO;
    }
    MF_TRY(mf_policy_create(0, out));
    return mf_policy_set_params(*out, w.data(), NPARAM);
}

// Runs a plain FP64 CG solve on m (b on the device) and, every
// `checkpoint_every` iterations, appends (features, label) samples of about
// one tile in `sample_stride` to the policy's training set.
mf_status mf_policy_collect(mf_learned p, mf_matrix m, const double *b, int checkpoint_every, int sample_stride,
                            long long max_samples, long long *samples_out)
{
    if (!p || !m || !b || checkpoint_every <= 0 || sample_stride <= 0) return MF_ERR_INVALID_ARG;
    if (m->v.rows != m->v.cols) return MF_ERR_INVALID_ARG;
    {
        float *bx;
        unsigned char *by;
        long long have;
        MF_TRY(policy_sample_buffers(p, max_samples, &bx, &by, &have));
    }
    double *x = nullptr;
    MF_CUDA(cudaMalloc(&x, sizeof(double) * (m->v.rows + 1)));
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    o.policy = MF_POLICY_FP64;
    o.tol = 1e-10;
    o.maxiter = 100000;
    mf_solve_report rep;
    memset(&rep, 0, sizeof(rep));
    CollectCtx ctx{p, sample_stride, (unsigned)(p->n * 2654435761ull)};
    TraceHook hook{checkpoint_every, collect_hook, &ctx};
    m->pol_have_prev = 0;
    mf_status st = cg_solve_traced(m, b, x, o, rep, &hook, 0);
    cudaFree(x);
    m->pol_have_prev = 0;
    if (samples_out) *samples_out = p->n;
    return (st == MF_ERR_NOT_CONVERGED) ? MF_OK : st;
}

mf_status mf_policy_label_counts(mf_learned p, long long counts[4])
{
    if (!p || !counts) return MF_ERR_INVALID_ARG;
    std::vector<unsigned char> y((size_t)p->n);
    if (p->n) MF_CUDA(cudaMemcpy(y.data(), p->d_y, (size_t)p->n, cudaMemcpyDeviceToHost));
    for (int k = 0; k < 4; k++) counts[k] = 0;
    for (unsigned char v : y) counts[v & 3]++;
    return MF_OK;
}

static mf_status grad_step(mf_learned p, const long long *d_idx, long long i0, int B, float lr, float *grad_host,
                           double *loss)
{
    const int nblk = (B + TB - 1) / TB;
    float *buf = nullptr;
    MF_CUDA(cudaMalloc(&buf, sizeof(float) * ((size_t)nblk * NPARAM + nblk + NPARAM)));
    float *gpart = buf, *lpart = buf + (size_t)nblk * NPARAM, *gout = lpart + nblk;
    const size_t smem = sizeof(float) * (NPARAM + 4 + (size_t)TB * SROW);
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mlp_grad<<<nblk, TB, smem>>>(p->d_w, p->d_x, p->d_y, d_idx, i0, B, 1.f / (float)B, gpart, lpart);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        if (lr > 0.f) p->steps++;
        k_mlp_update<<<grid_for4(NPARAM, 256), 256>>>(nblk, gpart, gout, p->d_master, p->d_m, p->d_v, p->d_w, lr,
                                                     p->steps);
        note_launch();
        e = cudaGetLastError();
    }
    std::vector<float> lp(nblk);
    if (e == cudaSuccess) e = cudaMemcpy(lp.data(), lpart, sizeof(float) * nblk, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grad_host) e = cudaMemcpy(grad_host, gout, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) {
        set_last_error("policy training step: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    double l = 0;
    for (float v : lp) l += v;
    if (loss) *loss = l / B;
    return MF_OK;
}

// Gradient of the mean cross-entropy loss of n given samples (host arrays)
// at the current BF16 weights; no update.
mf_status mf_policy_eval_grad(mf_learned p, const float *X, const int *Y, int n, float *grad, double *loss)
{
    if (!p || !X || !Y || n <= 0 || !grad) return MF_ERR_INVALID_ARG;
    float *ox = p->d_x;
    unsigned char *oy = p->d_y;
    float *dx = nullptr;
    unsigned char *dy = nullptr;
    MF_CUDA(cudaMalloc(&dx, sizeof(float) * NF * (size_t)n));
    MF_CUDA(cudaMalloc(&dy, (size_t)n + 16));
    std::vector<unsigned char> y8(n);
    for (int i = 0; i < n; i++) y8[i] = (unsigned char)(Y[i] & 3);
    cudaMemcpy(dx, X, sizeof(float) * NF * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(dy, y8.data(), (size_t)n, cudaMemcpyHostToDevice);
    p->d_x = dx;
    p->d_y = dy;
    mf_status st = grad_step(p, nullptr, 0, n, 0.f, grad, loss);
    p->d_x = ox;
    p->d_y = oy;
    cudaFree(dx);
    cudaFree(dy);
    return st;
}

// Adam training over the collected samples: `epochs` passes in a seeded
// shuffled order, minibatches of `batch` samples.
mf_status mf_policy_train(mf_learned p, int epochs, int batch, float lr, uint64_t seed, double *loss_first,
                          double *loss_last)
{
    if (!p || epochs <= 0 || batch <= 0 || lr <= 0 || p->n == 0) return MF_ERR_INVALID_ARG;
    const long long n = p->n;
    std::vector<long long> idx((size_t)n);
    long long *d_idx = nullptr;
    MF_CUDA(cudaMalloc(&d_idx, sizeof(long long) * (size_t)n));
    double first = -1, last = 0;
    for (int e = 0; e < epochs; e++) {
        for (long long i = 0; i < n; i++) idx[(size_t)i] = i;
        for (long long i = n - 1; i > 0; i--) {
            const long long j = (long long)(mix64(seed + (uint64_t)e * 0x9E3779B97F4A7C15ull + (uint64_t)i) % (uint64_t)(i + 1));
            std::swap(idx[(size_t)i], idx[(size_t)j]);
        }
        cudaMemcpy(d_idx, idx.data(), sizeof(long long) * (size_t)n, cudaMemcpyHostToDevice);
        double sum = 0;
        long long cnt = 0;
        for (long long i0 = 0; i0 + batch <= n || (i0 < n && i0 == 0); i0 += batch) {
            const int B = (int)std::min<long long>(batch, n - i0);
            double l = 0;
            mf_status st = grad_step(p, d_idx, i0, B, lr, nullptr, &l);
            if (st != MF_OK) {
                cudaFree(d_idx);
                return st;
            }
            if (first < 0) first = l;
            sum += l * B;
            cnt += B;
        }
        last = cnt ? sum / cnt : 0;
    }
    cudaFree(d_idx);
    if (loss_first) *loss_first = first;
    if (loss_last) *loss_last = last;
    return MF_OK;
}

mf_status mf_matrix_attach_policy(mf_matrix m, mf_learned p)
{
    if (!m) return MF_ERR_INVALID_ARG;
    m->policy = p;
    m->policy_loaded = p ? 1 : 0;
    m->pol_have_prev = 0;
    return MF_OK;
}

}  // extern "C"
