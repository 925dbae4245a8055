// bicgstab.cu -- the persistent BiCGSTAB solver kernel (FP64 and mixed).
//
// The reference runs 50 unpreconditioned BiCGSTAB iterations inside one
// persistent kernel with two SpMVs, five atomic dot products and four
// grid-wide waits per iteration (src/Mille-feuille-bicg.h:202-474, 478-822,
// 826-1185; mixed precision with separate classes for p and s in
// src/main-bicg-mixed.cu:122-723).  Here one cooperative launch runs the
// loop to the tolerance with three grid-wide reductions per iteration:
//   v = A p    with p = r + beta (p_old - omega v_old) formed on the fly;
//   (rhat.v)                                   -> alpha
//   t = A s    with s = r - alpha v formed on the fly;
//   (t.s, t.t)                                 -> omega
//   x += alpha p + omega s, r = s - omega t;
//   (rhat.r, r.r)                              -> beta, convergence
// p and v are double-buffered so no pass has to finish writing them before
// the next SpMV starts.  Mixed precision follows the CG solver: packed
// per-tile classes, FP32 vectors and accumulation, FP64 dot products and
// FP64 reliable updates of the residual.  On staged chunks (LAY 2, mixed)
// each SpMV copies two vectors into shared memory: the update pass, which
// knows omega, stores w = p - omega v (one rounding, as the on-the-fly form)
// over p, so the next p = r + beta w needs r and w only.
#include <algorithm>
#include <type_traits>

#include "persist.cuh"

namespace mf {
namespace {
using namespace persist;

template <class SM>
__device__ __forceinline__ void grid_sum2(const CgArgs &a, double l0, double l1, int slot, GridCtx &gc, SM &S,
                                          double &o0, double &o1)
{
    const int G = gridDim.x;
    const double c0 = block_sum<NT>(l0, S.warp);
    const double c1 = block_sum<NT>(l1, S.warp);
    if (threadIdx.x == 0) {
        a.partials[slot * G + blockIdx.x] = c0;
        a.partials[(slot + 1) * G + blockIdx.x] = c1;
    }
    gc.epoch++;
    gc.ok = gc.ok && MF_GRID_BARRIER(a.bar, gc.epoch, a.status, a.budget_ns);
    o0 = block_sum_partials<NT>(a.partials + slot * G, G, S.warp);
    o1 = block_sum_partials<NT>(a.partials + (slot + 1) * G, G, S.warp);
}

#ifndef MF_STAGED_MINB_BICG
#define MF_STAGED_MINB_BICG 4
#endif

template <bool MIX, int LAY>
struct BicgSmem {
    using type = typename std::conditional<
        LAY == 0, SolverSmem, typename std::conditional<LAY == 1, SlotSmem, StagedSmem<MIX>>::type>::type;
};

template <bool MIX, int LAY>
__global__ void __launch_bounds__(NT, LAY == 0 ? MINB : LAY == 1 ? SMINB : MF_STAGED_MINB_BICG) k_bicgstab(CgArgs a)
{
    using VT = typename VecT<MIX>::T;
    using SM = typename BicgSmem<MIX, LAY>::type;
    static_assert(LAY != 2 || MIX, "staged BiCGSTAB is the mixed kernel");
    constexpr int PK = MIX ? 1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &S = *reinterpret_cast<SM *>(smem_raw);
    const MfTiles &A = a.A;
    const int g = blockIdx.x;
    const int sb0 = a.part[g], se0 = a.part[g + 1];
    const int cb = LAY == 0 ? a.cta_chunk[g] : a.scta_chunk[g], ce = LAY == 0 ? a.cta_chunk[g + 1] : a.scta_chunk[g + 1];
    const int row0 = sb0 * MF_TILE, row1 = min(se0 * MF_TILE, A.rows);
    VT *r = (VT *)a.r, *rh = (VT *)a.rhat, *t = (VT *)a.t, *xlo = (VT *)a.xlo;
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

    double rho, beta, nb, rmax, alpha, omega;
    int it, refs;
    if (a.start) {
        double lb = 0.0, lr = 0.0;
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            const double bv = a.b[i];
            const VT rv = (VT)bv;
            a.xhi[i] = 0.0;
            r[i] = rv;
            rh[i] = rv;
            ((VT *)a.p0)[i] = (VT)0;
            ((VT *)a.v0)[i] = (VT)0;
            if (MIX) xlo[i] = (VT)0;
            lb = __dadd_rn(lb, __dmul_rn(bv, bv));
            lr = __dadd_rn(lr, __dmul_rn((double)rv, (double)rv));
        }
        double bb, rr0;
        grid_sum2(a, lb, lr, 0, gc, S, bb, rr0);
        nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
        rho = rr0;  // rhat = r0
        beta = 0.0;
        alpha = 1.0;
        omega = 1.0;
        rmax = sqrt(rr0);
        it = 0;
        refs = 0;
        st[S_RELRES] = sqrt(rr0) / nb;
    } else {
        rho = st[S_RHO];
        beta = st[S_BETA];
        nb = st[S_NB];
        rmax = st[S_RMAX];
        it = (int)st[S_ITERS];
        refs = (int)st[S_REFS];
        alpha = st[S_ALPHA];
        omega = st[S_OMEGA];
    }
    int exit_reason = EXIT_MAXITER;
    double rnorm = a.start ? rmax : st[S_RELRES] * nb;
    double relres_true = rnorm / nb;
    while (gc.ok) {
        // an exactly zero residual ends a fixed-count run too
        if ((!a.fixed && rnorm <= a.tol * nb) || rnorm == 0.0) {
            exit_reason = EXIT_CONVERGED;
            break;
        }
        if (it >= a.maxiter) {
            exit_reason = EXIT_MAXITER;
            break;
        }
        const VT *pold = (const VT *)((it & 1) ? a.p1 : a.p0);
        VT *pnew = (VT *)((it & 1) ? a.p0 : a.p1);
        const VT *vold = (const VT *)((it & 1) ? a.v1 : a.v0);
        VT *vnew = (VT *)((it & 1) ? a.v0 : a.v1);
        const VT bt = (VT)beta, om = (VT)omega;
        const VT *rr = r;
        // ---- v = A p, p = r + beta (p_old - omega v_old) ----
        // (staged: p_old already holds w = p_old - omega v_old)
        auto psrc = [=](int c) -> VT {
            if constexpr (LAY == 2) return fmaf(bt, pold[c], rr[c]);
            else if constexpr (MIX) return fmaf(bt, fmaf(-om, vold[c], pold[c]), rr[c]);
            else return fma(bt, fma(-om, vold[c], pold[c]), rr[c]);
        };
        double loc = 0.0;
        auto aout = [&](int s, int rw, auto y, auto xown, bool has_own) {
            const int i = s * MF_TILE + rw;
            const VT pn = has_own ? (VT)xown : psrc(i);
            const VT vi = (VT)y;
            pnew[i] = pn;
            vnew[i] = vi;
            loc = __dadd_rn(loc, __dmul_rn((double)rh[i], (double)vi));
        };
        if constexpr (LAY == 2) {
            if (!spmv_staged<PK, true, VT, 2>(a, S, gc, cb, ce, rr, pold, bt, aout, nullptr)) gc.ok = false;
        } else {
            if (!spmv_any<PK, LAY>(a, S, gc, cb, ce, sb0, se0, psrc, aout, nullptr)) gc.ok = false;
        }
        double rv, dummy;
        grid_sum2(a, loc, 0.0, 2, gc, S, rv, dummy);
        if (!gc.ok) break;
        if (!(rv != 0.0) || !isfinite(rv)) {
            if (g == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        alpha = rho / rv;
        const VT al = (VT)alpha;
        const VT *vn = vnew;
        // ---- t = A s, s = r - alpha v ----
        auto ssrc = [=](int c) -> VT {
            if constexpr (MIX) return fmaf(-al, vn[c], rr[c]);
            else return fma(-al, vn[c], rr[c]);
        };
        double lts = 0.0, ltt = 0.0;
        auto tout = [&](int s, int rw, auto y, auto xown, bool has_own) {
            const int i = s * MF_TILE + rw;
            const VT si = has_own ? (VT)xown : ssrc(i);
            const VT ti = (VT)y;
            t[i] = ti;
            lts = __dadd_rn(lts, __dmul_rn((double)ti, (double)si));
            ltt = __dadd_rn(ltt, __dmul_rn((double)ti, (double)ti));
        };
        if constexpr (LAY == 2) {
            if (!spmv_staged<PK, true, VT, 2>(a, S, gc, cb, ce, rr, vn, (VT)-al, tout, nullptr)) gc.ok = false;
        } else {
            if (!spmv_any<PK, LAY>(a, S, gc, cb, ce, sb0, se0, ssrc, tout, nullptr)) gc.ok = false;
        }
        double ts, tt;
        grid_sum2(a, lts, ltt, 4, gc, S, ts, tt);
        if (!gc.ok) break;
        omega = (tt != 0.0) ? ts / tt : 0.0;
        const VT omn = (VT)omega;
        // ---- x += alpha p + omega s, r = s - omega t ----
        double lrh = 0.0, lrr = 0.0;
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            const VT si = ssrc(i);
            const VT ri = MIX ? (VT)fmaf((float)-omn, (float)t[i], (float)si) : (VT)fma(-(double)omn, (double)t[i], (double)si);
            if (MIX) {
                xlo[i] = fmaf((float)omn, (float)si, fmaf((float)al, (float)pnew[i], (float)xlo[i]));
                // staged: w = p - omega v, read by the next first SpMV
                if (LAY == 2) pnew[i] = (VT)fmaf(-(float)omn, (float)vnew[i], (float)pnew[i]);
            } else {
                a.xhi[i] = fma(omega, (double)si, fma(alpha, (double)pnew[i], a.xhi[i]));
            }
            r[i] = ri;
            lrh = __dadd_rn(lrh, __dmul_rn((double)rh[i], (double)ri));
            lrr = __dadd_rn(lrr, __dmul_rn((double)ri, (double)ri));
        }
        double rho_new, rrn;
        grid_sum2(a, lrh, lrr, 6, gc, S, rho_new, rrn);
        if (!gc.ok) break;
        it++;
        rnorm = sqrt(rrn);
        if (MIX && (rnorm <= a.delta * rmax || (!a.fixed && rnorm <= a.tol * nb))) {
            // ---- reliable update: x_hi += x_lo; r = b - A x_hi in FP64 ----
            for (int i = row0 + threadIdx.x; i < row1; i += NT) {
                const double xn = a.xhi[i] + (double)xlo[i];
                a.xhi[i] = xn;
                if (LAY == 2) a.xs[i] = xn;  // padded copy the staged SpMV reads
                xlo[i] = (VT)0;
            }
            grid_sync(a, gc);
            if (!gc.ok) break;
            double l1 = 0.0, l2 = 0.0;
            const double *xh = a.xhi;
            auto xsrc = [=](int c) -> double { return xh[c]; };
            auto rout = [&](int s, int rw, double y, auto, bool) {
                const int i = s * MF_TILE + rw;
                const VT rv2 = (VT)(a.b[i] - y);
                r[i] = rv2;
                l1 = __dadd_rn(l1, __dmul_rn((double)rh[i], (double)rv2));
                l2 = __dadd_rn(l2, __dmul_rn((double)rv2, (double)rv2));
            };
            if constexpr (LAY == 2) {
                if (!spmv_staged<0, false, double, 1>(a, S, gc, cb, ce, (const double *)a.xs, (const double *)nullptr,
                                                      0.0, rout, nullptr))
                    gc.ok = false;
            } else {
                if (!spmv_any<0, LAY>(a, S, gc, cb, ce, sb0, se0, xsrc, rout, nullptr)) gc.ok = false;
            }
            grid_sum2(a, l1, l2, 0, gc, S, rho_new, rrn);
            if (!gc.ok) break;
            rnorm = sqrt(rrn);
            rmax = rnorm;
            refs++;
        }
        relres_true = rnorm / nb;
        if (!(omega != 0.0) || !isfinite(rho_new)) {
            if (rnorm <= a.tol * nb && !a.fixed) {
                exit_reason = EXIT_CONVERGED;
                rho = rho_new;
                break;
            }
            if (g == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        if (a.hist && g == 0 && threadIdx.x == 0) a.hist[it] = rnorm / nb;
    }
    if (MIX && exit_reason != EXIT_CHECKPOINT && gc.ok) {
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            a.xhi[i] = a.xhi[i] + (double)xlo[i];
            xlo[i] = (VT)0;
        }
    }
    if (g == 0 && threadIdx.x == 0) {
        st[S_RHO] = rho;
        st[S_BETA] = beta;
        st[S_NB] = nb;
        st[S_RMAX] = rmax;
        st[S_ITERS] = (double)it;
        st[S_REFS] = (double)refs;
        st[S_EXIT] = (double)exit_reason;
        st[S_RELRES] = relres_true;
        st[S_ALPHA] = alpha;
        st[S_OMEGA] = omega;
    }
}

template <bool MIX, int LAY>
int max_ctas_bicg()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t dyn = sizeof(typename BicgSmem<MIX, LAY>::type);
        cudaFuncSetAttribute(k_bicgstab<MIX, LAY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bicgstab<MIX, LAY>, NT, dyn);
        cached = sms * (per > 0 ? per : 1);
    }
    return cached;
}

}  // namespace

int bicgstab_grid(mf_matrix m, bool mixed, int layout)
{
    const bool slots = layout != 0;
    int maxc = layout == 2   ? max_ctas_bicg<true, 2>()  // mixed only
               : layout == 1 ? (mixed ? max_ctas_bicg<true, 1>() : max_ctas_bicg<false, 1>())
                             : (mixed ? max_ctas_bicg<true, 0>() : max_ctas_bicg<false, 0>());
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

mf_status launch_bicgstab(bool mixed, CgArgs &a, int G, cudaStream_t s)
{
    void *args[] = {&a};
    note_launch();
    const void *fn;
    size_t dyn;
    if (a.spos && mixed) {
        dyn = sizeof(StagedSmem<true>);
        max_ctas_bicg<true, 2>(), fn = (const void *)k_bicgstab<true, 2>;
    } else if (a.sslot) {
        dyn = sizeof(SlotSmem);
        if (mixed) max_ctas_bicg<true, 1>(), fn = (const void *)k_bicgstab<true, 1>;
        else max_ctas_bicg<false, 1>(), fn = (const void *)k_bicgstab<false, 1>;
    } else {
        dyn = sizeof(SolverSmem);
        if (mixed) max_ctas_bicg<true, 0>(), fn = (const void *)k_bicgstab<true, 0>;
        else max_ctas_bicg<false, 0>(), fn = (const void *)k_bicgstab<false, 0>;
    }
    MF_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(NT), args, dyn, s));
    return MF_OK;
}

}  // namespace mf
