// cg.cu -- the persistent CG solver kernel (FP64 and mixed precision).
//
// The reference runs CG inside one persistent kernel whose warps sync through
// atomic counters and spin-waits, with atomicAdd(double) dot products
// (src/Mille-feuille-cg.h:168-350, 352-580, 1109-1343; mixed precision in
// src/main-cg-mixed.cu:99-468, 998-1377).  This kernel keeps that shape --
// one launch runs the whole iteration loop -- and changes how it maps to a
// B200:
//   * cooperative launch sized to the resident CTAs, so every grid-wide wait
//     can finish; every wait is bounded and reports MF_ERR_TIMEOUT;
//   * each CTA owns a contiguous, cost-balanced range of 16-row strips, both
//     for the SpMV and for the vector updates; a half-warp stages one strip
//     (payload, column bytes, row pointers, x segments) in shared memory with
//     asynchronous 16-byte copies before computing its 16 rows;
//   * two grid-wide reductions per iteration and no third barrier: the new
//     search direction p = r + beta p is formed on the fly while the SpMV
//     gathers its x segments (p is double-buffered), so no pass writes p
//     before the next SpMV may read it;
//   * deterministic dot products (fixed per-thread order, fixed CTA tree,
//     per-CTA partials summed in the same order by every CTA);
//   * mixed precision (policies STATIC/RULE/LEARNED): per-tile payload classes
//     fp32/fp16/int8/bypass packed per strip, FP32 vectors and FP32
//     accumulation, FP64 dot products, and reliable updates: when ||r|| fell
//     by refine_delta, the FP32 correction is added to the FP64 solution and
//     r is replaced by the FP64 true residual b - A x computed from the FP64
//     payload.  Convergence is only declared on that FP64 true residual.
#include <cstdlib>

#include "strip_stage.cuh"
#include "solver.h"

namespace mf {
namespace {

constexpr int NT = 256;

template <bool MIX>
struct VecT {
    using T = double;
};
template <>
struct VecT<true> {
    using T = float;
};

struct GridCtx {
    unsigned long long epoch;
    bool ok;
};

__device__ __forceinline__ double grid_sum(const CgArgs &a, double local, int slot, GridCtx &gc, double *s_warp,
                                           double *s_res)
{
    const int G = gridDim.x;
    double cta = block_sum<NT>(local, s_warp);
    if (threadIdx.x == 0) a.partials[slot * G + blockIdx.x] = cta;
    gc.epoch++;
    gc.ok = gc.ok && grid_barrier(a.bar, gc.epoch * (unsigned long long)G, a.status, a.budget_ns);
    if (threadIdx.x < 32) {
        double s = warp_sum_partials(a.partials + slot * G, G);
        if (threadIdx.x == 0) *s_res = s;
    }
    __syncthreads();
    return *s_res;
}

__device__ __forceinline__ void grid_sync(const CgArgs &a, GridCtx &gc)
{
    gc.epoch++;
    gc.ok = gc.ok && grid_barrier(a.bar, gc.epoch * (unsigned long long)gridDim.x, a.status, a.budget_ns);
}

// Stage strip bi: metadata into lanes, payload/column/row-pointer bytes into
// shared memory.  PK 0: FP64 canonical payload; PK 1: packed mixed payload.
template <int PK>
__device__ __forceinline__ StripMeta stage_strip(const CgArgs &a, StripBuf &sb, int bi, int hl)
{
    const MfTiles &A = a.A;
    StripMeta m;
    m.t0 = A.tile_ptr[bi];
    const int t1 = A.tile_ptr[bi + 1];
    m.cnt = t1 - m.t0;
    m.e0 = A.tile_nnz[m.t0];
    const int e1 = A.tile_nnz[t1];
    m.staged = (m.cnt <= STAGE_MAXT) && (e1 - m.e0 <= STAGE_CAPE);
    m.my_tc = 0;
    m.my_off = 0;
    m.my_nz = 0;
    m.my_pb = 0;
    m.my_cls = MF_CLASS_FP64;
    long long pb_abs = 0;
    if (hl < m.cnt) {
        const int t = m.t0 + hl;
        m.my_tc = A.tile_columnidx[t];
        const int o = A.tile_nnz[t];
        m.my_off = o - m.e0;
        m.my_nz = A.tile_nnz[t + 1] - o;
        if (PK == 1) {
            pb_abs = (long long)a.poff[t];
            m.my_cls = a.wcls[t];
        } else {
            pb_abs = 8ll * o;
        }
    }
    if (!m.staged) return m;
    long long pbase;
    if (PK == 1)
        pbase = stage_range(sb.pay, a.pay, a.poff[m.t0], a.poff[t1], hl);
    else
        pbase = stage_range(sb.pay, (const unsigned char *)A.val, 8ll * m.e0, 8ll * e1, hl);
    m.my_pb = (int)(pb_abs - pbase);
    const long long cbase = stage_range(sb.col, A.col, m.e0, e1, hl);
    // keep the column base in my_off (entries are addressed relative to it)
    m.my_off += (int)(m.e0 - cbase);
    const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
    const long long pr0 = A.rows_multiple_of_16 ? 16ll * m.t0 : (long long)A.csrptr_offset[m.t0];
    const long long pbase2 = stage_range(sb.ptr, A.ptr, pr0, pr0 + (long long)m.cnt * rowlen, hl);
    // ptr of tile j, row r lives at sb.ptr[pshift + j*rowlen + r]
    sb.pshift = (int)(pr0 - pbase2);
    return m;
}

// Row r of a staged strip: sum over tiles in column order of the sequential
// per-tile row sums.  FP64 mode: rounded separately (bit-identical to
// blockspmv_cpu); mixed: FP32 fused multiply-add accumulation.
template <int PK>
__device__ __forceinline__ double staged_row(const StripBuf &sb, const StripMeta &m, int hl, unsigned hmask,
                                             int rowlen)
{
    double accd = 0.0;
    float accf = 0.0f;
    for (int j = 0; j < m.cnt; j++) {
        const int off = __shfl_sync(hmask, m.my_off, j, 16);
        const int nz = __shfl_sync(hmask, m.my_nz, j, 16);
        const int pb = __shfl_sync(hmask, m.my_pb, j, 16);
        const int cls = __shfl_sync(hmask, m.my_cls, j, 16);
        if (hl >= rowlen) continue;
        const int pj = sb.pshift + j * rowlen;
        const int lo = sb.ptr[pj + hl];
        const int hi = (hl == rowlen - 1) ? nz : (int)sb.ptr[pj + hl + 1];
        const double *seg = sb.seg[j];
        if (PK == 0) {
            const double *v = (const double *)(sb.pay + pb);
            double s = 0.0;
            for (int k = lo; k < hi; k++) s = __dadd_rn(s, __dmul_rn(seg[sb.col[off + k]], v[k]));
            accd = __dadd_rn(accd, s);
        } else {
            float s = 0.0f;
            if (cls == MF_CLASS_FP32 || cls == MF_CLASS_FP64) {
                const float *v = (const float *)(sb.pay + pb);
                for (int k = lo; k < hi; k++) s = fmaf(v[k], (float)seg[sb.col[off + k]], s);
            } else if (cls == MF_CLASS_FP16) {
                const __half *v = (const __half *)(sb.pay + pb);
                for (int k = lo; k < hi; k++) s = fmaf(__half2float(v[k]), (float)seg[sb.col[off + k]], s);
            } else if (cls == MF_CLASS_INT8) {
                const int8_t *v = (const int8_t *)(sb.pay + pb);
                for (int k = lo; k < hi; k++) s = fmaf((float)v[k], (float)seg[sb.col[off + k]], s);
            }
            accf += s;
        }
    }
    return PK == 0 ? accd : (double)accf;
}

// Direct (unstaged) row for strips above the staging caps; same order.
template <int PK, class Src>
__device__ __forceinline__ double direct_row(const CgArgs &a, int bi, int r, int rowlen, Src src)
{
    const MfTiles &A = a.A;
    const int t0 = A.tile_ptr[bi], t1 = A.tile_ptr[bi + 1];
    double accd = 0.0;
    float accf = 0.0f;
    for (int t = t0; t < t1; t++) {
        const int off = A.tile_nnz[t], nz = A.tile_nnz[t + 1] - off;
        const int xo = A.tile_columnidx[t] * MF_TILE;
        const int po = A.rows_multiple_of_16 ? t * MF_TILE : A.csrptr_offset[t];
        const int lo = A.ptr[po + r];
        const int hi = (r == rowlen - 1) ? nz : (int)A.ptr[po + r + 1];
        if (PK == 0) {
            double s = 0.0;
            for (int k = lo; k < hi; k++) s = __dadd_rn(s, __dmul_rn((double)src(xo + A.col[off + k]), A.val[off + k]));
            accd = __dadd_rn(accd, s);
        } else {
            const int cls = a.wcls[t];
            const unsigned char *pb = a.pay + a.poff[t];
            float s = 0.0f;
            for (int k = lo; k < hi; k++) {
                float v = 0.0f;
                if (cls == MF_CLASS_FP32 || cls == MF_CLASS_FP64) v = ((const float *)pb)[k];
                else if (cls == MF_CLASS_FP16) v = __half2float(((const __half *)pb)[k]);
                else if (cls == MF_CLASS_INT8) v = (float)((const int8_t *)pb)[k];
                else break;
                s = fmaf(v, (float)src(xo + A.col[off + k]), s);
            }
            accf += s;
        }
    }
    return PK == 0 ? accd : (double)accf;
}

// One strip's 16 rows of y = A src (src: functor giving the x value of a
// column).  Returns row hl's value (0 for lanes past rowlen).
template <int PK, class Src>
__device__ __forceinline__ double strip_product(const CgArgs &a, StripBuf &sb, int bi, int hl, unsigned hmask,
                                                Src src)
{
    const MfTiles &A = a.A;
    const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
    StripMeta m = stage_strip<PK>(a, sb, bi, hl);
    if (!m.staged) {
        __syncwarp(hmask);
        return (hl < rowlen) ? direct_row<PK>(a, bi, hl, rowlen, src) : 0.0;
    }
    // x segments: lane hl computes element hl of every tile's 16-column segment
    for (int j = 0; j < m.cnt; j++) {
        const int tc = __shfl_sync(hmask, m.my_tc, j, 16);
        const int c = tc * MF_TILE + hl;
        sb.seg[j][hl] = (c < A.cols) ? (double)src(c) : 0.0;
    }
    cp_async_wait_all();
    __syncwarp(hmask);
    const double y = staged_row<PK>(sb, m, hl, hmask, rowlen);
    __syncwarp(hmask);
    return y;
}

template <bool MIX>
__global__ void __launch_bounds__(NT, 4) k_cg(CgArgs a)
{
    using VT = typename VecT<MIX>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_warp[NT / 32];
    __shared__ double s_res;
    StripBuf *bufs = (StripBuf *)smem_raw;
    const MfTiles &A = a.A;
    const int sb0 = a.part[blockIdx.x], se0 = a.part[blockIdx.x + 1];
    const int lane = threadIdx.x & 31, hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
    const unsigned hmask = (lane < 16) ? 0x0000ffffu : 0xffff0000u;
    StripBuf &sb = bufs[hw];
    const int hstep = NT / MF_TILE;
    VT *r = (VT *)a.r, *q = (VT *)a.q, *xlo = (VT *)a.xlo;
    GridCtx gc{0ull, true};
    double *st = a.state;

    double rho, beta, nb, rmax;
    int it, refs;
    if (a.start) {
        double lb = 0.0, lr = 0.0;
        for (int bi = sb0 + hw; bi < se0; bi += hstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (hl < rowlen) {
                const int i = bi * MF_TILE + hl;
                const double bv = a.b[i];
                const VT rv = (VT)bv;
                a.xhi[i] = 0.0;
                r[i] = rv;
                ((VT *)a.p0)[i] = (VT)0;
                if (MIX) xlo[i] = (VT)0;
                lb = __dadd_rn(lb, __dmul_rn(bv, bv));
                lr = __dadd_rn(lr, __dmul_rn((double)rv, (double)rv));
            }
        }
        const double bb = grid_sum(a, lb, 0, gc, s_warp, &s_res);
        rho = MIX ? grid_sum(a, lr, 1, gc, s_warp, &s_res) : bb;
        nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
        beta = 0.0;
        rmax = sqrt(rho);
        it = 0;
        refs = 0;
        if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[0] = sqrt(bb) / nb;
    } else {
        rho = st[S_RHO];
        beta = st[S_BETA];
        nb = st[S_NB];
        rmax = st[S_RMAX];
        it = (int)st[S_ITERS];
        refs = (int)st[S_REFS];
    }
    int exit_reason = EXIT_MAXITER;
    double relres_true = sqrt(rho) / nb;
    // optional phase timers (thread 0 of each CTA)
    unsigned long long tph[5] = {0, 0, 0, 0, 0}, tmark = 0;
    const bool timed = a.timing != nullptr && threadIdx.x == 0;
#define MF_MARK(k)                                        \
    if (timed) {                                          \
        const unsigned long long now_ = globaltimer_ns(); \
        if ((k) >= 0) tph[(k)] += now_ - tmark;           \
        tmark = now_;                                     \
    }
    bool converged_check = false;
    while (gc.ok) {
        if (!a.fixed && sqrt(rho) <= a.tol * nb) {
            exit_reason = EXIT_CONVERGED;
            break;
        }
        if (it >= a.maxiter) {
            exit_reason = EXIT_MAXITER;
            break;
        }
        const VT *pold = (const VT *)((it & 1) ? a.p1 : a.p0);
        VT *pnew = (VT *)((it & 1) ? a.p0 : a.p1);
        const VT bt = (VT)beta;
        MF_MARK(-1);
        // ---- q = A p_new with p_new = r + beta p_old formed on the fly ----
        double loc = 0.0;
        auto psrc = [=](int c) -> VT {
            if constexpr (MIX) return fmaf(bt, pold[c], r[c]);
            else return fma(bt, pold[c], r[c]);
        };
        for (int bi = sb0 + hw; bi < se0; bi += hstep) {
            const double y = strip_product<MIX ? 1 : 0>(a, sb, bi, hl, hmask, psrc);
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (hl < rowlen) {
                const int i = bi * MF_TILE + hl;
                const VT pn = psrc(i);
                const VT qi = (VT)y;
                pnew[i] = pn;
                q[i] = qi;
                loc = __dadd_rn(loc, __dmul_rn((double)pn, (double)qi));
            }
        }
        MF_MARK(0);
        const double pq = grid_sum(a, loc, 2, gc, s_warp, &s_res);
        MF_MARK(1);
        if (!gc.ok) break;
        if (!(pq != 0.0) || !isfinite(pq)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        const double alpha = rho / pq;
        // ---- x += alpha p, r -= alpha q ----
        loc = 0.0;
        for (int bi = sb0 + hw; bi < se0; bi += hstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (hl < rowlen) {
                const int i = bi * MF_TILE + hl;
                if (MIX) {
                    xlo[i] = fmaf((float)alpha, (float)pnew[i], (float)xlo[i]);
                    const float ri = fmaf(-(float)alpha, (float)q[i], (float)r[i]);
                    r[i] = ri;
                    loc = __dadd_rn(loc, __dmul_rn((double)ri, (double)ri));
                } else {
                    a.xhi[i] = fma(alpha, (double)pnew[i], a.xhi[i]);
                    const double ri = fma(-alpha, (double)q[i], (double)r[i]);
                    r[i] = ri;
                    loc = __dadd_rn(loc, __dmul_rn(ri, ri));
                }
            }
        }
        MF_MARK(2);
        double rho_new = grid_sum(a, loc, 3, gc, s_warp, &s_res);
        MF_MARK(3);
        if (!gc.ok) break;
        it++;
        bool refined = false;
        if (MIX && (sqrt(rho_new) <= a.delta * rmax || (!a.fixed && sqrt(rho_new) <= a.tol * nb))) {
            // ---- reliable update: x_hi += x_lo; r = b - A x_hi in FP64 ----
            for (int bi = sb0 + hw; bi < se0; bi += hstep) {
                const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
                if (hl < rowlen) {
                    const int i = bi * MF_TILE + hl;
                    a.xhi[i] = a.xhi[i] + (double)xlo[i];
                    xlo[i] = (VT)0;
                }
            }
            grid_sync(a, gc);
            if (!gc.ok) break;
            loc = 0.0;
            const double *xh = a.xhi;
            auto xsrc = [=](int c) -> double { return xh[c]; };
            for (int bi = sb0 + hw; bi < se0; bi += hstep) {
                const double y = strip_product<0>(a, sb, bi, hl, hmask, xsrc);
                const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
                if (hl < rowlen) {
                    const int i = bi * MF_TILE + hl;
                    const double rt = a.b[i] - y;
                    const VT rv = (VT)rt;
                    r[i] = rv;
                    loc = __dadd_rn(loc, __dmul_rn((double)rv, (double)rv));
                }
            }
            rho_new = grid_sum(a, loc, 1, gc, s_warp, &s_res);
            if (!gc.ok) break;
            rmax = sqrt(rho_new);
            relres_true = sqrt(rho_new) / nb;
            refs++;
            refined = true;
            MF_MARK(4);
        }
        beta = rho_new / rho;
        rho = rho_new;
        if (!MIX) relres_true = sqrt(rho) / nb;
        if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[it] = sqrt(rho) / nb;
        if (refined && a.exit_on_refine) {
            exit_reason = EXIT_CHECKPOINT;
            converged_check = true;
            break;
        }
    }
    (void)converged_check;
    if (MIX && exit_reason != EXIT_CONVERGED && exit_reason != EXIT_CHECKPOINT && gc.ok) {
        // leaving with an unflushed FP32 correction: fold it into x
        for (int bi = sb0 + hw; bi < se0; bi += hstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (hl < rowlen) {
                const int i = bi * MF_TILE + hl;
                a.xhi[i] = a.xhi[i] + (double)xlo[i];
                xlo[i] = (VT)0;
            }
        }
    }
#undef MF_MARK
    if (timed)
        for (int k = 0; k < 5; k++) a.timing[blockIdx.x * 8 + k] += tph[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[S_RHO] = rho;
        st[S_BETA] = beta;
        st[S_NB] = nb;
        st[S_RMAX] = rmax;
        st[S_ITERS] = (double)it;
        st[S_REFS] = (double)refs;
        st[S_EXIT] = (double)exit_reason;
        st[S_RELRES] = relres_true;
    }
}

// ||b - A x||^2 and ||b||^2 from y = A x, deterministic: per-CTA partials,
// then one CTA sums them in a fixed tree.
__global__ void k_resid_partials(int n, const double *__restrict__ b, const double *__restrict__ ax,
                                 double *__restrict__ part)
{
    __shared__ double s_warp[8];
    double rr = 0.0, bb = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = b[i] - ax[i];
        rr += d * d;
        bb += b[i] * b[i];
    }
    double s1 = block_sum<256>(rr, s_warp);
    double s2 = block_sum<256>(bb, s_warp);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s1;
        part[2 * blockIdx.x + 1] = s2;
    }
}

__global__ void k_resid_final(int nblk, const double *__restrict__ part, double *__restrict__ out)
{
    __shared__ double s_warp[8];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    a = block_sum<256>(a, s_warp);
    b = block_sum<256>(b, s_warp);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
    }
}

template <bool MIX>
int max_ctas_for()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t dyn = sizeof(StripBuf) * (NT / MF_TILE);
        cudaFuncSetAttribute(k_cg<MIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg<MIX>, NT, dyn);
        cached = sms * (per > 0 ? per : 1);
    }
    return cached;
}

}  // namespace

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

mf_status solver_resources(mf_matrix m, int G, SolverWork &w)
{
    const size_t n = (size_t)m->v.tilem * MF_TILE + 16;
    size_t off = 0;
    const size_t o_r = off; off += align256(n * 8);
    const size_t o_p0 = off; off += align256(n * 8);
    const size_t o_p1 = off; off += align256(n * 8);
    const size_t o_q = off; off += align256(n * 8);
    const size_t o_xlo = off; off += align256(n * 8);
    const size_t o_ax = off; off += align256(n * 8);
    const size_t o_part = off; off += align256((size_t)4 * G * 8);
    const size_t o_rp = off; off += align256((size_t)2 * 1024 * 8);
    const size_t o_out = off; off += align256(8 * 8);
    const size_t o_state = off; off += align256(32 * 8);
    const size_t o_tim = off; off += align256((size_t)G * 8 * 8);
    const size_t o_bar = off; off += align256(8);
    const size_t o_st = off; off += align256(8);
    MF_TRY(ensure_work(m, off));
    char *base = (char *)m->work;
    w.r = base + o_r;
    w.p0 = base + o_p0;
    w.p1 = base + o_p1;
    w.q = base + o_q;
    w.xlo = base + o_xlo;
    w.ax = (double *)(base + o_ax);
    w.partials = (double *)(base + o_part);
    w.rpart = (double *)(base + o_rp);
    w.out = (double *)(base + o_out);
    w.state = (double *)(base + o_state);
    w.timing = (unsigned long long *)(base + o_tim);
    w.bar = (unsigned long long *)(base + o_bar);
    w.status = (int *)(base + o_st);
    return MF_OK;
}

int solver_grid(mf_matrix m, bool mixed)
{
    int maxc = mixed ? max_ctas_for<true>() : max_ctas_for<false>();
    if (const char *e = getenv("MF_SOLVER_CTAS")) {
        const int v = atoi(e);
        if (v > 0 && v < maxc) maxc = v;
    }
    int want = ceil_div(m->v.tilem, NT / MF_TILE);
    if (want < 1) want = 1;
    return want < maxc ? want : maxc;
}

mf_status true_residual(mf_matrix m, const double *b, const double *x, SolverWork &w, double *relres, cudaStream_t s)
{
    const int n = m->v.rows;
    MF_TRY(spmv_fp64(m->v, x, w.ax, s));
    const int nblk = 512;
    k_resid_partials<<<nblk, 256, 0, s>>>(n, b, w.ax, w.rpart);
    note_launch();
    MF_CUDA(cudaGetLastError());
    k_resid_final<<<1, 256, 0, s>>>(nblk, w.rpart, w.out + 4);
    note_launch();
    MF_CUDA(cudaGetLastError());
    double h[2];
    MF_CUDA(cudaMemcpyAsync(h, w.out + 4, sizeof(h), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    *relres = h[1] > 0 ? sqrt(h[0]) / sqrt(h[1]) : sqrt(h[0]);
    return MF_OK;
}

mf_status launch_cg(bool mixed, CgArgs &a, int G, cudaStream_t s)
{
    const size_t dyn = sizeof(StripBuf) * (NT / MF_TILE);
    void *args[] = {&a};
    note_launch();
    if (mixed) {
        max_ctas_for<true>();
        MF_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg<true>, dim3(G), dim3(NT), args, dyn, s));
    } else {
        max_ctas_for<false>();
        MF_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg<false>, dim3(G), dim3(NT), args, dyn, s));
    }
    return MF_OK;
}

}  // namespace mf
