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
#include <cuda_fp16.h>

#include <cstdlib>

#include "solver.h"
#include "tma.cuh"

namespace mf {
namespace {

constexpr int NT = CH_STRIPS * MF_TILE;  // one half-warp per strip of a chunk
#ifndef MF_CG_MINB
#define MF_CG_MINB 3
#endif
constexpr int MINB = MF_CG_MINB;  // CTAs per SM the registers allow
constexpr int RECS = 64;                    // chunk records cached in shared memory

// Byte layout of one shared-memory stage (every region 16-byte aligned,
// sized for the largest 16-byte-rounded range it receives).
constexpr int OFF_TPTR = 0;                                   // tile_ptr[s0..s1]
constexpr int OFF_TCOL = 112;                                 // tile_columnidx[t0..t1)
constexpr int OFF_TNNZ = OFF_TCOL + CH_TILES * 4 + 32;        // tile_nnz[t0..t1]
constexpr int OFF_POFF = OFF_TNNZ + CH_TILES * 4 + 48;        // packed offsets[t0..t1]
constexpr int OFF_WCLS = OFF_POFF + CH_TILES * 4 + 48;        // classes[t0..t1)
constexpr int OFF_PTR = OFF_WCLS + CH_TILES + 32;             // u8 row pointers
constexpr int OFF_COL = OFF_PTR + CH_TILES * MF_TILE + 32;    // in-tile column bytes
constexpr int OFF_PAY = OFF_COL + CH_ENTRIES + 32;            // payload
constexpr int STAGE_BYTES = OFF_PAY + CH_ENTRIES * 8 + 32;
static_assert(OFF_TNNZ % 16 == 0 && OFF_POFF % 16 == 0 && OFF_WCLS % 16 == 0 && OFF_PTR % 16 == 0 &&
                  OFF_COL % 16 == 0 && OFF_PAY % 16 == 0 && STAGE_BYTES % 16 == 0,
              "stage regions must be 16-byte aligned");

struct StageHdr {
    ChunkRec rec;
    int sh_tptr, sh_tcol, sh_tnnz, sh_poff, sh_wcls, sh_ptr, sh_col, sh_pay;
};

struct __align__(16) SolverSmem {
    unsigned char stage[2][STAGE_BYTES];
    double seg[CH_TILES * MF_TILE];
    StageHdr hdr[2];
    ChunkRec recs[RECS];
    uint64_t bar[2];
    double warp[NT / 32];
    double res;
};

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
    unsigned use[2];  // completed uses of each stage (mbarrier phase parity)
};

__device__ __forceinline__ double grid_sum(const CgArgs &a, double local, int slot, GridCtx &gc, SolverSmem &S)
{
    const int G = gridDim.x;
    double cta = block_sum<NT>(local, S.warp);
    if (threadIdx.x == 0) a.partials[slot * G + blockIdx.x] = cta;
    gc.epoch++;
    gc.ok = gc.ok && grid_barrier_sharded(a.bar, gc.epoch, a.status, a.budget_ns);
    if (threadIdx.x < 32) {
        double s = warp_sum_partials(a.partials + slot * G, G);
        if (threadIdx.x == 0) S.res = s;
    }
    __syncthreads();
    return S.res;
}

__device__ __forceinline__ void grid_sync(const CgArgs &a, GridCtx &gc)
{
    gc.epoch++;
    gc.ok = gc.ok && grid_barrier_sharded(a.bar, gc.epoch, a.status, a.budget_ns);
}

// Offset of tile t's u8 row pointers in Blockcsr_Ptr (csrptr_offset without
// a memory access: every tile has 16 pointers except those of a short last
// strip).
__device__ __forceinline__ long long ptr_off(const CgArgs &a, int t)
{
    return (t < a.last_tile_begin) ? 16ll * t
                                   : 16ll * a.last_tile_begin + (long long)(t - a.last_tile_begin) * a.last_rowlen;
}

__device__ __forceinline__ void add_range(unsigned char *dst, const unsigned char *src, long long a0, long long a1,
                                          uint64_t *bar, int &shift)
{
    const long long c0 = a0 & ~15ll, c1 = (a1 + 15) & ~15ll;
    shift = (int)(a0 - c0);
    if (c1 > c0) bulk_g2s_hint(dst, src + c0, (unsigned)(c1 - c0), bar, l2_policy_evict_first());
}

__device__ __forceinline__ unsigned range_bytes(long long a0, long long a1)
{
    const long long c0 = a0 & ~15ll, c1 = (a1 + 15) & ~15ll;
    return (unsigned)(c1 - c0);
}

// Thread 0: stage chunk c into stage k.
template <int PK>
__device__ void issue_chunk(const CgArgs &a, SolverSmem &S, int c, int k)
{
    const int cb = a.cta_chunk[blockIdx.x];
    const ChunkRec r = (c - cb < RECS) ? S.recs[c - cb] : a.chunks[c];
    StageHdr &h = S.hdr[k];
    h.rec = r;
    unsigned char *st = S.stage[k];
    const MfTiles &A = a.A;
    // expected bytes first (the barrier counts them down as copies land)
    unsigned total = range_bytes(4ll * r.s0, 4ll * (r.s1 + 1));
    if (!r.direct) {
        total += range_bytes(4ll * r.t0, 4ll * r.t1) + range_bytes(4ll * r.t0, 4ll * (r.t1 + 1));
        total += range_bytes(ptr_off(a, r.t0), ptr_off(a, r.t1)) + range_bytes(r.e0, r.e1);
        if (PK == 1) {
            total += range_bytes(4ll * r.t0, 4ll * (r.t1 + 1)) + range_bytes(r.t0, r.t1) + range_bytes(r.y0, r.y1);
        } else {
            total += range_bytes(8ll * r.e0, 8ll * r.e1);
        }
    }
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.bar[k], total);
    add_range(st + OFF_TPTR, (const unsigned char *)A.tile_ptr, 4ll * r.s0, 4ll * (r.s1 + 1), &S.bar[k], h.sh_tptr);
    if (r.direct) return;
    add_range(st + OFF_TCOL, (const unsigned char *)A.tile_columnidx, 4ll * r.t0, 4ll * r.t1, &S.bar[k], h.sh_tcol);
    add_range(st + OFF_TNNZ, (const unsigned char *)A.tile_nnz, 4ll * r.t0, 4ll * (r.t1 + 1), &S.bar[k], h.sh_tnnz);
    add_range(st + OFF_PTR, A.ptr, ptr_off(a, r.t0), ptr_off(a, r.t1), &S.bar[k], h.sh_ptr);
    add_range(st + OFF_COL, A.col, r.e0, r.e1, &S.bar[k], h.sh_col);
    if (PK == 1) {
        add_range(st + OFF_POFF, (const unsigned char *)a.poff, 4ll * r.t0, 4ll * (r.t1 + 1), &S.bar[k], h.sh_poff);
        add_range(st + OFF_WCLS, a.wcls, r.t0, r.t1, &S.bar[k], h.sh_wcls);
        add_range(st + OFF_PAY, a.pay, r.y0, r.y1, &S.bar[k], h.sh_pay);
    } else {
        add_range(st + OFF_PAY, (const unsigned char *)A.val, 8ll * r.e0, 8ll * r.e1, &S.bar[k], h.sh_pay);
    }
}

// Row r of strip s from a staged chunk (reference order: tiles in column
// order, each tile's row entries in order).  FP64 payload: products and sums
// rounded separately (bit-identical to blockspmv_cpu); packed payload: FP32
// fused multiply-add accumulation.  The walk advances pointers tile by tile
// so that each tile costs a handful of shared-memory loads.
template <int PK>
__device__ __forceinline__ double chunk_row(const CgArgs &a, const SolverSmem &S, int k, int s, int r, int rowlen,
                                            double &xown, bool &has_own)
{
    const StageHdr &h = S.hdr[k];
    const ChunkRec &rec = h.rec;
    const unsigned char *st = S.stage[k];
    const int *tp = (const int *)(st + OFF_TPTR + h.sh_tptr);
    const int ja = tp[s - rec.s0] - rec.t0, jb = tp[s - rec.s0 + 1] - rec.t0;
    const int *tn = (const int *)(st + OFF_TNNZ + h.sh_tnnz) + ja;
    const int *tcl = (const int *)(st + OFF_TCOL + h.sh_tcol) + ja;
    const unsigned char *cb = st + OFF_COL + h.sh_col - rec.e0;
    // row pointers of tile ja; every tile has `rowlen` pointers in a strip
    const unsigned char *prow = st + OFF_PTR + h.sh_ptr + (ptr_off(a, rec.t0 + ja) - ptr_off(a, rec.t0)) + r;
    const double *seg = S.seg + ja * MF_TILE;
    const unsigned char *payb = st + OFF_PAY + h.sh_pay;
    const unsigned *po = (const unsigned *)(st + OFF_POFF + h.sh_poff) + ja;
    const unsigned char *wc = st + OFF_WCLS + h.sh_wcls + ja;
    const bool last = (r == rowlen - 1);
    double accd = 0.0;
    float accf = 0.0f;
    has_own = false;
    int o0 = tn[0];
    for (int j = 0; j < jb - ja; j++) {
        const int o1 = tn[j + 1];
        const int lo = prow[0];
        const int hi = last ? (o1 - o0) : (int)prow[1];
        if (!has_own && tcl[j] == s) {  // diagonal tile: its segment holds this row's x value
            xown = seg[r];
            has_own = true;
        }
        const unsigned char *cl = cb + o0;
        if (PK == 0) {
            const double *v = (const double *)payb + (o0 - rec.e0);
            double sm = 0.0;
            for (int q = lo; q < hi; q++) sm = __dadd_rn(sm, __dmul_rn(seg[cl[q]], v[q]));
            accd = __dadd_rn(accd, sm);
        } else {
            const int cls = wc[j];
            const unsigned char *vb = payb + (po[j] - rec.y0);
            float sm = 0.0f;
            if (cls == MF_CLASS_FP32 || cls == MF_CLASS_FP64) {
                const float *v = (const float *)vb;
                for (int q = lo; q < hi; q++) sm = fmaf(v[q], (float)seg[cl[q]], sm);
            } else if (cls == MF_CLASS_FP16) {
                const __half *v = (const __half *)vb;
                for (int q = lo; q < hi; q++) sm = fmaf(__half2float(v[q]), (float)seg[cl[q]], sm);
            } else if (cls == MF_CLASS_INT8) {
                const int8_t *v = (const int8_t *)vb;
                for (int q = lo; q < hi; q++) sm = fmaf((float)v[q], (float)seg[cl[q]], sm);
            }
            accf += sm;
        }
        o0 = o1;
        prow += rowlen;
        seg += MF_TILE;
    }
    return PK == 0 ? accd : (double)accf;
}

// Row r of strip s straight from global memory (chunks flagged direct).
template <int PK, class Src>
__device__ double direct_row(const CgArgs &a, int s, int r, int rowlen, Src src)
{
    const MfTiles &A = a.A;
    const int t0 = A.tile_ptr[s], t1 = A.tile_ptr[s + 1];
    double accd = 0.0;
    float accf = 0.0f;
    for (int t = t0; t < t1; t++) {
        const int off = A.tile_nnz[t], nz = A.tile_nnz[t + 1] - off;
        const int xo = A.tile_columnidx[t] * MF_TILE;
        const long long po = ptr_off(a, t);
        const int lo = A.ptr[po + r];
        const int hi = (r == rowlen - 1) ? nz : (int)A.ptr[po + r + 1];
        if (PK == 0) {
            double sm = 0.0;
            for (int q = lo; q < hi; q++)
                sm = __dadd_rn(sm, __dmul_rn((double)src(xo + A.col[off + q]), A.val[off + q]));
            accd = __dadd_rn(accd, sm);
        } else {
            const int cls = a.wcls[t];
            const unsigned char *vb = a.pay + a.poff[t];
            float sm = 0.0f;
            for (int q = lo; q < hi; q++) {
                float v;
                if (cls == MF_CLASS_FP32 || cls == MF_CLASS_FP64) v = ((const float *)vb)[q];
                else if (cls == MF_CLASS_FP16) v = __half2float(((const __half *)vb)[q]);
                else if (cls == MF_CLASS_INT8) v = (float)((const int8_t *)vb)[q];
                else break;
                sm = fmaf(v, (float)src(xo + A.col[off + q]), sm);
            }
            accf += sm;
        }
    }
    return PK == 0 ? accd : (double)accf;
}

// y = A src over this CTA's chunks [cb, ce); out(s, r, y) receives every row.
// Returns false when a bounded wait expired (status set).
template <int PK, class Src, class Out>
__device__ bool spmv_chunks(const CgArgs &a, SolverSmem &S, GridCtx &gc, int cb, int ce, Src src, Out &out,
                            unsigned long long *tph)
{
    const bool timed = tph != nullptr && threadIdx.x == 0;
    unsigned long long tm = timed ? globaltimer_ns() : 0ull;
#define MF_SUB(k)                                          \
    if (timed) {                                           \
        const unsigned long long nw_ = globaltimer_ns();   \
        tph[(k)] += nw_ - tm;                              \
        tm = nw_;                                          \
    }
    const MfTiles &A = a.A;
    const int tid = threadIdx.x, hw = tid >> 4, hl = tid & 15;
    if (tid == 0) {
        if (cb < ce) issue_chunk<PK>(a, S, cb, 0);
        if (cb + 1 < ce) issue_chunk<PK>(a, S, cb + 1, 1);
    }
    __syncthreads();
    bool ok = true;
    for (int c = cb; c < ce; c++) {
        const int k = (c - cb) & 1;
        if (!mbar_wait_bounded(&S.bar[k], gc.use[k] & 1u, a.status, a.budget_ns)) {
            ok = false;
            // the other stage may still have a copy in flight: wait for it
            // (bounded) before leaving so no copy lands in freed memory
            if (c + 1 < ce) mbar_wait_bounded(&S.bar[k ^ 1], gc.use[k ^ 1] & 1u, a.status, a.budget_ns);
            break;
        }
        gc.use[k]++;
        MF_SUB(5);
        const ChunkRec &rec = S.hdr[k].rec;
        if (rec.direct) {
            const int s = rec.s0;
            const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
            if (hw == 0 && hl < rowlen) out(s, hl, direct_row<PK>(a, s, hl, rowlen, src), 0.0, false);
        } else {
            const int nt = rec.t1 - rec.t0;
            const int *tc = (const int *)(S.stage[k] + OFF_TCOL + S.hdr[k].sh_tcol);
            // x segments: gathers issued SEGB at a time before any is used
            constexpr int SEGB = 4;
            for (int v0 = tid; v0 < nt * MF_TILE; v0 += NT * SEGB) {
                decltype(src(0)) sv[SEGB];
#pragma unroll
                for (int u = 0; u < SEGB; u++) {
                    const int v = v0 + u * NT;
                    const int col = (v < nt * MF_TILE) ? tc[v >> 4] * MF_TILE + (v & 15) : A.cols;
                    sv[u] = (col < A.cols) ? src(col) : (decltype(src(0)))0;
                }
#pragma unroll
                for (int u = 0; u < SEGB; u++) {
                    const int v = v0 + u * NT;
                    if (v < nt * MF_TILE) S.seg[v] = (double)sv[u];
                }
            }
            __syncthreads();
            MF_SUB(6);
            const int s = rec.s0 + hw;
            if (s < rec.s1) {
                const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
                if (hl < rowlen) {
                    double xown = 0.0;
                    bool has_own = false;
                    const double y = chunk_row<PK>(a, S, k, s, hl, rowlen, xown, has_own);
                    out(s, hl, y, xown, has_own);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && c + 2 < ce) issue_chunk<PK>(a, S, c + 2, k);
        MF_SUB(7);
    }
#undef MF_SUB
    return ok;
}

template <bool MIX>
__global__ void __launch_bounds__(NT, MINB) k_cg(CgArgs a)
{
    using VT = typename VecT<MIX>::T;
    constexpr int PK = MIX ? 1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolverSmem &S = *reinterpret_cast<SolverSmem *>(smem_raw);
    const MfTiles &A = a.A;
    const int g = blockIdx.x;
    const int sb0 = a.part[g], se0 = a.part[g + 1];
    const int cb = a.cta_chunk[g], ce = a.cta_chunk[g + 1];
    const int row0 = sb0 * MF_TILE, row1 = min(se0 * MF_TILE, A.rows);
    VT *r = (VT *)a.r, *q = (VT *)a.q, *xlo = (VT *)a.xlo;
    GridCtx gc;
    gc.epoch = 0;
    gc.ok = true;
    gc.use[0] = gc.use[1] = 0;
    double *st = a.state;
    if (threadIdx.x == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        mbar_fence_init();
    }
    for (int c = cb + threadIdx.x; c < ce && c - cb < RECS; c += NT) S.recs[c - cb] = a.chunks[c];
    __syncthreads();

    double rho, beta, nb, rmax;
    int it, refs;
    if (a.start) {
        double lb = 0.0, lr = 0.0;
        for (int i = row0 + threadIdx.x; i < row1; i += NT) {
            const double bv = a.b[i];
            const VT rv = (VT)bv;
            a.xhi[i] = 0.0;
            r[i] = rv;
            ((VT *)a.p0)[i] = (VT)0;
            if (MIX) xlo[i] = (VT)0;
            lb = __dadd_rn(lb, __dmul_rn(bv, bv));
            lr = __dadd_rn(lr, __dmul_rn((double)rv, (double)rv));
        }
        const double bb = grid_sum(a, lb, 0, gc, S);
        rho = MIX ? grid_sum(a, lr, 1, gc, S) : bb;
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
        const VT *rr = r;
        auto psrc = [=](int c) -> VT {
            if constexpr (MIX) return fmaf(bt, pold[c], rr[c]);
            else return fma(bt, pold[c], rr[c]);
        };
        MF_MARK(-1);
        // ---- q = A p_new, p_new = r + beta p_old formed on the fly ----
        double loc = 0.0;
        auto aout = [&](int s, int rw, double y, double xown, bool has_own) {
            const int i = s * MF_TILE + rw;
            const VT pn = has_own ? (VT)xown : psrc(i);
            const VT qi = (VT)y;
            pnew[i] = pn;
            q[i] = qi;
            loc = __dadd_rn(loc, __dmul_rn((double)pn, (double)qi));
        };
        if (!spmv_chunks<PK>(a, S, gc, cb, ce, psrc, aout, timed ? tph : nullptr)) gc.ok = false;
        MF_MARK(0);
        const double pq = grid_sum(a, loc, 2, gc, S);
        MF_MARK(1);
        if (!gc.ok) break;
        if (!(pq != 0.0) || !isfinite(pq)) {
            if (g == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            exit_reason = EXIT_BREAKDOWN;
            break;
        }
        const double alpha = rho / pq;
        // ---- x += alpha p, r -= alpha q over this CTA's rows ----
        loc = 0.0;
        {
            constexpr int U = 4;
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
                    } else {
                        a.xhi[i] = fma(alpha, (double)pv[u], (double)xv[u]);
                        const double ri = fma(-alpha, (double)qv[u], (double)rv[u]);
                        r[i] = ri;
                        loc = __dadd_rn(loc, __dmul_rn(ri, ri));
                    }
                }
            }
        }
        MF_MARK(2);
        double rho_new = grid_sum(a, loc, 3, gc, S);
        MF_MARK(3);
        if (!gc.ok) break;
        it++;
        bool refined = false;
        if (MIX && (sqrt(rho_new) <= a.delta * rmax || (!a.fixed && sqrt(rho_new) <= a.tol * nb))) {
            // ---- reliable update: x_hi += x_lo; r = b - A x_hi in FP64 ----
            for (int i = row0 + threadIdx.x; i < row1; i += NT) {
                a.xhi[i] = a.xhi[i] + (double)xlo[i];
                xlo[i] = (VT)0;
            }
            grid_sync(a, gc);
            if (!gc.ok) break;
            loc = 0.0;
            const double *xh = a.xhi;
            auto xsrc = [=](int c) -> double { return xh[c]; };
            auto rout = [&](int s, int rw, double y, double, bool) {
                const int i = s * MF_TILE + rw;
                const VT rv = (VT)(a.b[i] - y);
                r[i] = rv;
                loc = __dadd_rn(loc, __dmul_rn((double)rv, (double)rv));
            };
            if (!spmv_chunks<0>(a, S, gc, cb, ce, xsrc, rout, nullptr)) gc.ok = false;
            rho_new = grid_sum(a, loc, 1, gc, S);
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
        if (a.hist && g == 0 && threadIdx.x == 0) a.hist[it] = sqrt(rho) / nb;
        if (refined && a.exit_on_refine) {
            exit_reason = EXIT_CHECKPOINT;
            break;
        }
    }
#undef MF_MARK
    if (MIX && exit_reason != EXIT_CONVERGED && exit_reason != EXIT_CHECKPOINT && gc.ok) {
        // leaving with an unflushed FP32 correction: fold it into x
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
        const size_t dyn = sizeof(SolverSmem);
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
    const size_t o_bar = off; off += align256(9 * 128);
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
    int want = ceil_div(m->v.tilem, CH_STRIPS);
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
    const size_t dyn = sizeof(SolverSmem);
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
