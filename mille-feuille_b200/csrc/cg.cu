// cg.cu -- the persistent CG solver kernel (FP64 and mixed precision).
//
// The reference runs CG inside one persistent kernel whose warps sync through
// atomic counters and spin-waits, with atomicAdd(double) dot products
// (src/Mille-feuille-cg.h:168-350, 352-580, 1109-1343; mixed precision in
// src/main-cg-mixed.cu:99-468, 998-1377).  This kernel keeps that shape --
// one launch runs the whole iteration loop -- and changes how it maps to a
// B200:
//   * cooperative launch sized to the resident CTAs, so every grid-wide wait
//     can finish; every wait (grid barrier, mbarrier) is bounded in time and
//     reports MF_ERR_TIMEOUT through a status word instead of hanging;
//   * each CTA owns a contiguous, cost-balanced range of 16-row strips, cut
//     into chunks of up to 16 strips.  A chunk's tile metadata, u8 row
//     pointers, column bytes and payload are contiguous byte ranges; one
//     thread stages them into shared memory with bulk asynchronous copies
//     (TMA, cp.async.bulk, completion on an mbarrier), two chunks in flight;
//     the CTA then builds the chunk's x segments and computes its rows from
//     shared memory, one half-warp per strip and one lane per row;
//   * two grid-wide reductions per iteration and no third barrier: the new
//     search direction p = r + beta p is formed while the SpMV builds its x
//     segments (p is double-buffered), so no pass must write p before the
//     next SpMV can start;
//   * deterministic dot products (fixed per-thread order, fixed CTA tree,
//     per-CTA partials summed in the same order by every CTA);
//   * mixed precision (policies STATIC/RULE/LEARNED): per-tile payload classes
//     fp32/fp16/int8/bypass packed per strip, FP32 vectors and FP32
//     accumulation, FP64 dot products, and reliable updates: when ||r|| fell
//     by refine_delta, the FP32 correction is added to the FP64 solution and
//     r is replaced by the FP64 true residual b - A x computed from the FP64
//     payload.  Convergence is only declared on that FP64 true residual.
#include <algorithm>
#include <type_traits>

#include "persist.cuh"

namespace mf {
namespace {
using namespace persist;

#ifndef MF_STAGED_MINB_MIX
#define MF_STAGED_MINB_MIX 4
#endif
#ifndef MF_STAGED_MINB_FP64
#define MF_STAGED_MINB_FP64 2
#endif
#ifndef MF_VEC_U
#define MF_VEC_U 4  // rows per thread in flight in the vector update pass
#endif
// CTAs per SM of the kernels on staged chunks (shared memory allows them)
constexpr int staged_minb(bool mix) { return mix ? MF_STAGED_MINB_MIX : MF_STAGED_MINB_FP64; }

template <bool MIX, int LAY>
struct CgSmem {
    using type = typename std::conditional<LAY == 0, SolverSmem,
                                           typename std::conditional<LAY == 1, SlotSmem, StagedSmem<MIX>>::type>::type;
};

// PC: Jacobi-preconditioned CG (z = D^-1 r; p = z + beta p; beta from r.z;
// convergence on ||r||), the same kernel otherwise.
template <bool MIX, int LAY, bool PC = false>
__global__ void __launch_bounds__(NT, LAY == 0 ? MINB : LAY == 1 ? SMINB : staged_minb(MIX)) k_cg(CgArgs a)
{
    using VT = typename VecT<MIX>::T;
    using SM = typename CgSmem<MIX, LAY>::type;
    constexpr int PK = MIX ? 1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &S = *reinterpret_cast<SM *>(smem_raw);
    const MfTiles &A = a.A;
    const int g = blockIdx.x;
    const int sb0 = a.part[g], se0 = a.part[g + 1];
    const int cb = LAY == 0 ? a.cta_chunk[g] : a.scta_chunk[g], ce = LAY == 0 ? a.cta_chunk[g + 1] : a.scta_chunk[g + 1];
    const int row0 = sb0 * MF_TILE, row1 = min(se0 * MF_TILE, A.rows);
    VT *r = (VT *)a.r, *q = (VT *)a.q, *xlo = (VT *)a.xlo;
    VT *z = (VT *)a.z;
    const double *dinv = a.dinv;
    GridCtx gc;
    gc.epoch = 0;
    gc.ok = true;
    gc.par = 0u;
    double *st = a.state;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (LAY == 0 ? 2 : NSTG); i++) mbar_init(&S.bar[i], LAY == 2 ? STAGED_ARRIVALS : 1);
        mbar_fence_init();
    }
    if constexpr (LAY == 0) {
        for (int c = cb + threadIdx.x; c < ce && c - cb < RECS; c += NT) S.recs[c - cb] = a.chunks[c];
    } else {
        constexpr int NREC = LAY == 1 ? SRECS : TRECS;
        for (int c = cb + threadIdx.x; c < ce && c - cb < NREC; c += NT) S.recs[c - cb] = a.schunks[c];
    }
    __syncthreads();

    double rho, beta, nb, rmax;
    double rz = 0.0;  // PC: r.z
    int it, refs;
    if (a.start) {
        double lb = 0.0, lr = 0.0, lz = 0.0;
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            const double bv = a.b[i];
            const VT rv = (VT)bv;
            a.xhi[i] = 0.0;
            r[i] = rv;
            ((VT *)a.p0)[i] = (VT)0;
            if (MIX) xlo[i] = (VT)0;
            if constexpr (PC) {
                const VT zv = (VT)(dinv[i] * (double)rv);
                z[i] = zv;
                lz = __dadd_rn(lz, __dmul_rn((double)rv, (double)zv));
            }
            lb = __dadd_rn(lb, __dmul_rn(bv, bv));
            lr = __dadd_rn(lr, __dmul_rn((double)rv, (double)rv));
        }
        const double bb = grid_sum(a, lb, 0, gc, S);
        rho = MIX ? grid_sum(a, lr, 1, gc, S) : bb;
        if constexpr (PC) rz = grid_sum(a, lz, 5, gc, S);
        nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
        beta = 0.0;
        rmax = sqrt(rho);
        it = 0;
        refs = 0;
        if (a.hist && g == 0 && threadIdx.x == 0) a.hist[0] = sqrt(bb) / nb;
    } else {
        rho = st[S_RHO];
        beta = st[S_BETA];
        nb = st[S_NB];
        rmax = st[S_RMAX];
        it = (int)st[S_ITERS];
        refs = (int)st[S_REFS];
        rz = st[S_RZ];
    }
    int exit_reason = EXIT_MAXITER;
    double relres_true = sqrt(rho) / nb;
    unsigned long long tph[8] = {0, 0, 0, 0, 0, 0, 0, 0}, tmark = 0;
    const bool timed = a.timing != nullptr && threadIdx.x == 0;
#define MF_MARK(k)                                        \
    if (timed) {                                          \
        const unsigned long long now_ = globaltimer_ns(); \
        if ((k) >= 0) tph[(k)] += now_ - tmark;           \
        tmark = now_;                                     \
    }
    while (gc.ok) {
        // an exactly zero residual ends a fixed-count run too (the next
        // step would divide 0 by 0)
        if ((!a.fixed && sqrt(rho) <= a.tol * nb) || rho == 0.0) {
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
        const VT *rr = PC ? z : r;  // p = rr + beta p_old (z when preconditioned)
        auto psrc = [=](int c) -> VT {
            if constexpr (MIX) return fmaf(bt, pold[c], rr[c]);
            else return fma(bt, pold[c], rr[c]);
        };
        MF_MARK(-1);
        // ---- q = A p_new, p_new = r + beta p_old formed on the fly ----
        double loc = 0.0;
        // y and xown: double, or float from the staged mixed SpMV (the same
        // values either way)
        auto aout = [&](int s, int rw, auto y, auto xown, bool has_own) {
            const int i = s * MF_TILE + rw;
            const VT pn = has_own ? (VT)xown : psrc(i);
            const VT qi = (VT)y;
            pnew[i] = pn;
            q[i] = qi;
            loc = __dadd_rn(loc, __dmul_rn((double)pn, (double)qi));
        };
        if constexpr (LAY == 2) {
            if (!spmv_staged<PK, true, VT, 2>(a, S, gc, cb, ce, rr, pold, bt, aout, timed ? tph : nullptr))
                gc.ok = false;
        } else {
            if (!spmv_any<PK, LAY>(a, S, gc, cb, ce, sb0, se0, psrc, aout, timed ? tph : nullptr)) gc.ok = false;
        }
        MF_MARK(0);
        const double pq = grid_sum(a, loc, 2, gc, S);
        MF_MARK(1);
        if (!gc.ok) break;
        if (!(pq != 0.0) || !isfinite(pq)) {
            if (g == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        const double alpha = (PC ? rz : rho) / pq;
        // ---- x += alpha p, r -= alpha q over this CTA's rows ----
        loc = 0.0;
        double locz = 0.0;  // PC: r.z
        {
            constexpr int U = MF_VEC_U;
            for (int i0 = row0 + threadIdx.x; i0 < row1; i0 += NT * U) {
                VT xv[U], pv[U], qv[U], rv[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int i = i0 + u * NT;
                    const bool in = i < row1;
                    xv[u] = in ? (MIX ? (VT)xlo[i] : (VT)a.xhi[i]) : (VT)0;
                    pv[u] = in ? pnew[i] : (VT)0;
                    qv[u] = in ? q[i] : (VT)0;
                    rv[u] = in ? r[i] : (VT)0;
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int i = i0 + u * NT;
                    if (i >= row1) break;
                    if constexpr (MIX) {
                        const float af = (float)alpha;
                        xlo[i] = fmaf(af, pv[u], xv[u]);
                        const float ri = fmaf(-af, qv[u], rv[u]);
                        r[i] = ri;
                        loc = __dadd_rn(loc, __dmul_rn((double)ri, (double)ri));
                        if constexpr (PC) {
                            const float zi = (float)(dinv[i] * (double)ri);
                            z[i] = zi;
                            locz = __dadd_rn(locz, __dmul_rn((double)ri, (double)zi));
                        }
                    } else {
                        a.xhi[i] = fma(alpha, (double)pv[u], (double)xv[u]);
                        const double ri = fma(-alpha, (double)qv[u], (double)rv[u]);
                        r[i] = ri;
                        loc = __dadd_rn(loc, __dmul_rn(ri, ri));
                        if constexpr (PC) {
                            const double zi = dinv[i] * ri;
                            z[i] = zi;
                            locz = __dadd_rn(locz, __dmul_rn(ri, zi));
                        }
                    }
                }
            }
        }
        MF_MARK(2);
        double rho_new, rz_new = 0.0;
        if constexpr (PC) grid_sum_pair(a, loc, locz, 3, gc, S, rho_new, rz_new);
        else rho_new = grid_sum(a, loc, 3, gc, S);
        MF_MARK(3);
        if (!gc.ok) break;
        it++;
        bool refined = false;
        if (MIX && (sqrt(rho_new) <= a.delta * rmax || (!a.fixed && sqrt(rho_new) <= a.tol * nb))) {
            // ---- reliable update: x_hi += x_lo; r = b - A x_hi in FP64 ----
            for (int i = row0 + threadIdx.x; i < row1; i += NT) {
                const double xn = a.xhi[i] + (double)xlo[i];
                a.xhi[i] = xn;
                if (LAY == 2) a.xs[i] = xn;  // padded copy the staged SpMV reads
                xlo[i] = (VT)0;
            }
            grid_sync(a, gc);
            if (!gc.ok) break;
            loc = 0.0;
            const double *xh = a.xhi;
            auto xsrc = [=](int c) -> double { return xh[c]; };
            locz = 0.0;
            auto rout = [&](int s, int rw, double y, auto, bool) {
                const int i = s * MF_TILE + rw;
                const VT rv = (VT)(a.b[i] - y);
                r[i] = rv;
                loc = __dadd_rn(loc, __dmul_rn((double)rv, (double)rv));
                if constexpr (PC) {
                    const VT zv = (VT)(dinv[i] * (double)rv);
                    z[i] = zv;
                    locz = __dadd_rn(locz, __dmul_rn((double)rv, (double)zv));
                }
            };
            if constexpr (LAY == 2) {
                if (!spmv_staged<0, false, double, 1>(a, S, gc, cb, ce, (const double *)a.xs, (const double *)nullptr,
                                                      0.0, rout, nullptr))
                    gc.ok = false;
            } else {
                if (!spmv_any<0, LAY>(a, S, gc, cb, ce, sb0, se0, xsrc, rout, nullptr)) gc.ok = false;
            }
            if constexpr (PC) grid_sum_pair(a, loc, locz, 0, gc, S, rho_new, rz_new);
            else rho_new = grid_sum(a, loc, 1, gc, S);
            if (!gc.ok) break;
            rmax = sqrt(rho_new);
            relres_true = sqrt(rho_new) / nb;
            refs++;
            refined = true;
            MF_MARK(4);
        }
        if constexpr (PC) {
            beta = rz_new / rz;
            rz = rz_new;
        } else {
            beta = rho_new / rho;
        }
        rho = rho_new;
        if (!MIX) relres_true = sqrt(rho) / nb;
        if (a.hist && g == 0 && threadIdx.x == 0) a.hist[it] = sqrt(rho) / nb;
        if ((refined && a.exit_on_refine) || (a.checkpoint_every > 0 && it % a.checkpoint_every == 0)) {
            exit_reason = EXIT_CHECKPOINT;
            break;
        }
    }
#undef MF_MARK
    if (MIX && exit_reason != EXIT_CHECKPOINT && gc.ok) {
        // fold any unflushed FP32 correction into x (zero after a refinement)
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            a.xhi[i] = a.xhi[i] + (double)xlo[i];
            xlo[i] = (VT)0;
        }
    }
    if (timed)
        for (int k = 0; k < 8; k++) a.timing[g * 8 + k] += tph[k];
    if (g == 0 && threadIdx.x == 0) {
        st[S_RHO] = rho;
        st[S_BETA] = beta;
        st[S_NB] = nb;
        st[S_RMAX] = rmax;
        st[S_ITERS] = (double)it;
        st[S_REFS] = (double)refs;
        st[S_EXIT] = (double)exit_reason;
        st[S_RELRES] = relres_true;
        st[S_RZ] = rz;
    }
}

// FP64 CG with one grid-wide reduction per iteration (the vector updates
// ride on the SpMV pass).  Pass k gathers p_k = r_{k-1} - alpha q_{k-1} +
// beta p_{k-1} on the fly from the previous pass's vectors (double-buffered
// r, q, p), computes q_k = A p_k, and for its own rows writes p_k, q_k,
// r_k = r_{k-1} - alpha q_{k-1} and x_k = x_{k-1} + alpha p_{k-1}; one
// reduction then gives p.q, r.q, q.q and r.r, from which alpha_k =
// (r.r)/(p.q) and the next ||r||^2 = r.r - 2 alpha r.q + alpha^2 q.q (so
// beta_k) follow without a second reduction.  In exact arithmetic this is the
// textbook method; the expanded ||r||^2 only feeds beta, the convergence test
// uses the explicit r.r.  Pass 0 starts from r = b, q = p = 0, alpha = beta
// = 0, so every pass runs the same code.  No checkpoints (the tracing and
// mixed-precision solves use k_cg).
template <int LAY>
__global__ void __launch_bounds__(NT, LAY == 0 ? MINB : SMINB) k_cg1(CgArgs a)
{
    using SM = typename std::conditional<LAY == 0, SolverSmem, SlotSmem>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &S = *reinterpret_cast<SM *>(smem_raw);
    const MfTiles &A = a.A;
    const int g = blockIdx.x;
    const int sb0 = a.part[g], se0 = a.part[g + 1];
    const int cb = LAY == 0 ? a.cta_chunk[g] : a.scta_chunk[g], ce = LAY == 0 ? a.cta_chunk[g + 1] : a.scta_chunk[g + 1];
    const int row0 = sb0 * MF_TILE, row1 = min(se0 * MF_TILE, A.rows);
    double *rb[2] = {(double *)a.r, (double *)a.rhat};
    double *qb[2] = {(double *)a.q, (double *)a.v0};
    double *pb[2] = {(double *)a.p0, (double *)a.p1};
    double *x = a.xhi;
    GridCtx gc;
    gc.epoch = 0;
    gc.ok = true;
    gc.par = 0u;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (LAY == 0 ? 2 : NSTG); i++) mbar_init(&S.bar[i], 1);
        mbar_fence_init();
    }
    if constexpr (LAY == 0) {
        for (int c = cb + threadIdx.x; c < ce && c - cb < RECS; c += NT) S.recs[c - cb] = a.chunks[c];
    } else {
        for (int c = cb + threadIdx.x; c < ce && c - cb < SRECS; c += NT) S.recs[c - cb] = a.schunks[c];
    }
    double lb = 0.0;
    for (int i = row0 + threadIdx.x; i < row1; i += NT) {
        const double bv = a.b[i];
        rb[0][i] = bv;
        qb[0][i] = 0.0;
        pb[0][i] = 0.0;
        x[i] = 0.0;
        lb = __dadd_rn(lb, __dmul_rn(bv, bv));
    }
    __syncthreads();
    const double bb = grid_sum(a, lb, 0, gc, S);
    const double nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
    if (a.hist && g == 0 && threadIdx.x == 0) a.hist[0] = sqrt(bb) / nb;
    double alpha = 0.0, beta = 0.0, rr = bb;
    int it = -1;  // updates done; pass 0 makes r_0
    int exit_reason = EXIT_MAXITER;
    while (gc.ok) {
        const int o = (it + 1) & 1;  // buffers of the previous pass
        const double *ro = rb[o], *qo = qb[o], *po = pb[o];
        double *rn = rb[o ^ 1], *qn = qb[o ^ 1], *pn = pb[o ^ 1];
        const double al = alpha, be = beta;
        auto psrc = [=](int c) -> double { return fma(be, po[c], fma(-al, qo[c], ro[c])); };
        double l[4] = {0.0, 0.0, 0.0, 0.0};  // p.q, r.q, q.q, r.r
        auto aout = [&](int s, int rw, double y, double xown, bool has_own) {
            const int i = s * MF_TILE + rw;
            const double pv = has_own ? xown : psrc(i);
            const double rv = fma(-al, qo[i], ro[i]);
            x[i] = fma(al, po[i], x[i]);
            pn[i] = pv;
            qn[i] = y;
            rn[i] = rv;
            l[0] = __dadd_rn(l[0], __dmul_rn(pv, y));
            l[1] = __dadd_rn(l[1], __dmul_rn(rv, y));
            l[2] = __dadd_rn(l[2], __dmul_rn(y, y));
            l[3] = __dadd_rn(l[3], __dmul_rn(rv, rv));
        };
        if (!spmv_any<0, LAY>(a, S, gc, cb, ce, sb0, se0, psrc, aout, nullptr)) gc.ok = false;
        double d[4];
        grid_sum4(a, l, 4, gc, S, d);
        if (!gc.ok) break;
        it++;
        rr = d[3];
        if (a.hist && g == 0 && threadIdx.x == 0) a.hist[it] = sqrt(rr) / nb;
        if ((!a.fixed && sqrt(rr) <= a.tol * nb) || rr == 0.0) {
            exit_reason = EXIT_CONVERGED;
            break;
        }
        if (it >= a.maxiter) {
            exit_reason = EXIT_MAXITER;
            break;
        }
        if (!(d[0] != 0.0) || !isfinite(d[0])) {
            if (g == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        alpha = rr / d[0];
        const double rr_next = rr - 2.0 * alpha * d[1] + alpha * alpha * d[2];
        beta = rr_next / rr;
    }
    if (g == 0 && threadIdx.x == 0) {
        double *st = a.state;
        st[S_RHO] = rr;
        st[S_BETA] = beta;
        st[S_NB] = nb;
        st[S_RMAX] = sqrt(rr);
        st[S_ITERS] = (double)(it < 0 ? 0 : it);
        st[S_REFS] = 0.0;
        st[S_EXIT] = (double)exit_reason;
        st[S_RELRES] = sqrt(rr) / nb;
    }
}

// Jacobi: 1 / a_ii of every row from the tile format (the diagonal tile of
// the row's strip, the row's entry in its column), 1 where the diagonal is
// missing or zero.
__global__ void k_jacobi_dinv(MfTiles A, double *__restrict__ dinv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.rows; i += gridDim.x * blockDim.x) {
        const int s = i >> 4, rw = i & 15;
        const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
        double d = 0.0;
        for (int t = A.tile_ptr[s]; t < A.tile_ptr[s + 1]; t++) {
            if (A.tile_columnidx[t] != s) continue;
            const int off = A.tile_nnz[t], nz = A.tile_nnz[t + 1] - off;
            const int po = A.csrptr_offset[t];
            const int lo = A.ptr[po + rw];
            const int hi = (rw == rowlen - 1) ? nz : (int)A.ptr[po + rw + 1];
            for (int q = lo; q < hi; q++)
                if (A.col[off + q] == rw) d = A.val[off + q];
            break;
        }
        dinv[i] = (d != 0.0) ? 1.0 / d : 1.0;
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

template <int LAY, bool MIX = false>
constexpr size_t smem_bytes()
{
    return sizeof(typename CgSmem<MIX, LAY>::type);
}

// The Jacobi variant of k_cg<MIX, LAY>: its shared-memory attribute set
// once, and whether as many of its CTAs are resident as of the plain one's
// (the grid is sized for those).
template <bool MIX, int LAY>
bool pc_ready(int G)
{
    static int resident = -1;
    if (resident < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t dyn = smem_bytes<LAY, MIX>();
        cudaFuncSetAttribute(k_cg<MIX, LAY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg<MIX, LAY, true>, NT, dyn);
        resident = sms * per;
    }
    return G <= resident;
}

template <bool MIX, int LAY>
int max_ctas_for()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t dyn = smem_bytes<LAY, MIX>();
        cudaFuncSetAttribute(k_cg<MIX, LAY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg<MIX, LAY>, NT, dyn);
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
    const size_t o_rhat = off; off += align256(n * 8);
    const size_t o_v0 = off; off += align256(n * 8);
    const size_t o_v1 = off; off += align256(n * 8);
    const size_t o_t = off; off += align256(n * 8);
    const size_t o_ax = off; off += align256(n * 8);
    const size_t o_part = off; off += align256((size_t)8 * G * 8);
    const size_t o_rp = off; off += align256((size_t)2 * 1024 * 8);
    const size_t o_out = off; off += align256(8 * 8);
    const size_t o_state = off; off += align256(32 * 8);
    const size_t o_tim = off; off += align256((size_t)G * 8 * 8);
    const size_t o_bar = off; off += align256(9 * 128);
    const size_t o_st = off; off += align256(8);
    MF_TRY(ensure_work(m, off));
    char *base = (char *)m->work;
    w.r = base + o_r;
    w.p0 = base + o_p0;
    w.p1 = base + o_p1;
    w.q = base + o_q;
    w.xlo = base + o_xlo;
    w.rhat = base + o_rhat;
    w.v0 = base + o_v0;
    w.v1 = base + o_v1;
    w.t = base + o_t;
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

int solver_grid(mf_matrix m, bool mixed, int layout)
{
    const bool slots = layout != 0;
    int maxc = layout == 2   ? (mixed ? max_ctas_for<true, 2>() : max_ctas_for<false, 2>())
               : layout == 1 ? (mixed ? max_ctas_for<true, 1>() : max_ctas_for<false, 1>())
                             : (mixed ? max_ctas_for<true, 0>() : max_ctas_for<false, 0>());
    if (const char *e = getenv("MF_SOLVER_CTAS")) {
        const int v = atoi(e);
        if (v > 0 && v < maxc) maxc = v;
    }
    int want = ceil_div(m->v.tilem, CH_STRIPS);
    // strips with long rows: enough CTAs for the slots, not only the strips
    if (slots && m->nslots > 0) want = std::max<long long>(want, (m->nslots + SC_SLOTS - 1) / SC_SLOTS);
    if (want < 1) want = 1;
    return want < maxc ? want : maxc;
}

mf_status jacobi_dinv(mf_matrix m, double *dinv, cudaStream_t s)
{
    if (m->v.rows == 0) return MF_OK;
    k_jacobi_dinv<<<std::min(ceil_div(m->v.rows, 256), 148 * 8), 256, 0, s>>>(m->v, dinv);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
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
    void *args[] = {&a};
    note_launch();
    const void *fn;
    size_t dyn;
    if (!mixed && a.one_reduction) {
        // the grid was sized for k_cg; k_cg1 runs when as many of its CTAs
        // are resident (same launch bounds, its own occupancy checked once)
        static int resident[2] = {-1, -1};
        const int li = a.sslot ? 1 : 0;
        dyn = a.sslot ? smem_bytes<1>() : smem_bytes<0>();
        fn = a.sslot ? (const void *)k_cg1<1> : (const void *)k_cg1<0>;
        if (resident[li] < 0) {
            int dev = 0, sms = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            MF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
            MF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, NT, dyn));
            resident[li] = sms * per;
        }
        if (G <= resident[li]) {
            MF_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(NT), args, dyn, s));
            return MF_OK;
        }
        a.one_reduction = 0;  // fall through to the two-reduction kernel
    }
    const bool pc = a.dinv != nullptr;
    bool ready = true;
    if (a.spos) {
        if (mixed) dyn = smem_bytes<2, true>(), max_ctas_for<true, 2>(),
                   fn = pc ? (ready = pc_ready<true, 2>(G), (const void *)k_cg<true, 2, true>) : (const void *)k_cg<true, 2>;
        else dyn = smem_bytes<2, false>(), max_ctas_for<false, 2>(),
             fn = pc ? (ready = pc_ready<false, 2>(G), (const void *)k_cg<false, 2, true>) : (const void *)k_cg<false, 2>;
    } else if (a.sslot) {
        dyn = smem_bytes<1>();
        if (mixed) max_ctas_for<true, 1>(),
            fn = pc ? (ready = pc_ready<true, 1>(G), (const void *)k_cg<true, 1, true>) : (const void *)k_cg<true, 1>;
        else max_ctas_for<false, 1>(),
            fn = pc ? (ready = pc_ready<false, 1>(G), (const void *)k_cg<false, 1, true>) : (const void *)k_cg<false, 1>;
    } else {
        dyn = smem_bytes<0>();
        if (mixed) max_ctas_for<true, 0>(),
            fn = pc ? (ready = pc_ready<true, 0>(G), (const void *)k_cg<true, 0, true>) : (const void *)k_cg<true, 0>;
        else max_ctas_for<false, 0>(),
            fn = pc ? (ready = pc_ready<false, 0>(G), (const void *)k_cg<false, 0, true>) : (const void *)k_cg<false, 0>;
    }
    if (!ready) {
        set_last_error("the Jacobi CG kernel cannot keep %d CTAs resident", G);
        return MF_ERR_UNSUPPORTED;
    }
    MF_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(NT), args, dyn, s));
    return MF_OK;
}

}  // namespace mf
