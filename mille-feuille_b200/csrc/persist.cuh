// persist.cuh -- building blocks shared by the persistent solver kernels
// (CG and BiCGSTAB): the shared-memory stage layout, TMA staging of a CTA's
// chunks of strips, the per-row products in the reference's summation order,
// and the deterministic grid-wide reductions.
#pragma once
#include <cuda_fp16.h>

#include <climits>
#include <cstdlib>
#include <type_traits>

#include "solver.h"
#include "tma.cuh"

namespace mf {
namespace persist {

constexpr int NT = CH_STRIPS * MF_TILE;  // one half-warp per strip of a chunk
#ifndef MF_CG_MINB
#define MF_CG_MINB 3
#endif
constexpr int MINB = MF_CG_MINB;  // CTAs per SM the registers allow
#ifndef MF_SLOT_MINB
#define MF_SLOT_MINB 3
#endif
#ifndef MF_SLOT_U
#define MF_SLOT_U 4
#endif
#ifndef MF_FLAT_BARRIER
#define MF_FLAT_BARRIER 1
#endif
#if MF_FLAT_BARRIER
#define MF_GRID_BARRIER grid_barrier_flat
#else
#define MF_GRID_BARRIER grid_barrier_fast
#endif
constexpr int SMINB = MF_SLOT_MINB;  // CTAs per SM of the row-slot kernels
constexpr int SLOT_U = MF_SLOT_U;    // slots loaded before any is used
constexpr int RECS = 64;                    // chunk records cached in shared memory

// Byte layout of one shared-memory stage (every region 16-byte aligned,
// sized for the largest 16-byte-rounded range it receives).
constexpr int OFF_TPTR = 0;                                   // tile_ptr[s0..s1]
constexpr int OFF_TCOL = ((CH_STRIPS + 1) * 4 + 32 + 15) / 16 * 16;  // tile_columnidx[t0..t1)
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

// Shared memory of the kernels that run from the row-slot layout: two
// stages, each holding one slot chunk (strip slot offsets, tile pointers,
// tile columns, slot words, then FP64 values or the mixed slot headers and
// payload).  Every region is 16-byte aligned and sized for the largest
// 16-byte-rounded range it receives.
constexpr int SOFF_SSLOT = 0;
constexpr int SOFF_TPTR = ((SC_STRIPS + 1) * 4 + 32 + 15) / 16 * 16;
constexpr int SOFF_TCOL = 2 * SOFF_TPTR;
constexpr int SOFF_META = SOFF_TCOL + SC_TILES * 4 + 32;
constexpr int SOFF_DATA = SOFF_META + SC_SLOTS * MF_TILE * 2 + 32;
constexpr int SOFF_PAY = SOFF_DATA + SC_SLOTS * 4 + 32;  // mixed payload after the slot headers
constexpr int SSTAGE_BYTES = SOFF_DATA + SC_SLOTS * MF_TILE * 8 + 32;
static_assert(SOFF_META % 16 == 0 && SOFF_DATA % 16 == 0 && SOFF_PAY % 16 == 0 && SSTAGE_BYTES % 16 == 0,
              "slot stage regions must be 16-byte aligned");
static_assert(SOFF_PAY + SC_SLOTS * 64 + 32 <= SSTAGE_BYTES, "mixed payload must fit the stage");

struct SlotHdr {
    SlotChunk rec;
    int sh_sslot, sh_tptr, sh_tcol, sh_meta, sh_data, sh_pay;
};

#ifndef MF_SLOT_STAGES
#define MF_SLOT_STAGES 2
#endif
constexpr int NSTG = MF_SLOT_STAGES;  // slot chunks in flight per CTA
constexpr int SRECS = 64;  // slot chunk records cached in shared memory

struct __align__(16) SlotSmem {
    unsigned char stage[NSTG][SSTAGE_BYTES];
    SlotHdr hdr[NSTG];
    SlotChunk recs[SRECS];
    double py[NT], px[NT];  // per-thread partial row sums / own p values (strips shared by half-warps)
    unsigned char pown[NT];
    uint64_t bar[NSTG];
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
    unsigned par;  // bit k: parity of the completed uses of stage k (its mbarrier phase)
};

template <class SM>
__device__ __forceinline__ double grid_sum(const CgArgs &a, double local, int slot, GridCtx &gc, SM &S)
{
    const int G = gridDim.x;
    double cta = block_sum<NT>(local, S.warp);
    if (threadIdx.x == 0) a.partials[slot * G + blockIdx.x] = cta;
    gc.epoch++;
    gc.ok = gc.ok && MF_GRID_BARRIER(a.bar, gc.epoch, a.status, a.budget_ns);
    return block_sum_partials<NT>(a.partials + slot * G, G, S.warp);
}

// Two sums at once (one barrier): slots slot and slot+1 of the partials;
// every CTA gets the same two values.  Consecutive reductions must use
// different slots (a CTA may write the next partials while another still
// reads these).
template <class SM>
__device__ __forceinline__ void grid_sum_pair(const CgArgs &a, double l0, double l1, int slot, GridCtx &gc, SM &S,
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

// Four sums at once (one barrier, one batch of partial loads): slots
// slot..slot+3 of the partials; every CTA gets the same four values.
template <class SM>
__device__ __forceinline__ void grid_sum4(const CgArgs &a, const double (&l)[4], int slot, GridCtx &gc, SM &S,
                                          double (&o)[4])
{
    const int G = gridDim.x;
    __shared__ double s_w4[NT / 32][4];
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = l[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    }
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; k++) s_w4[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double c = 0.0;
            for (int i = 0; i < NT / 32; i++) c += s_w4[i][k];
            a.partials[(slot + k) * G + blockIdx.x] = c;
        }
    }
    gc.epoch++;
    gc.ok = gc.ok && MF_GRID_BARRIER(a.bar, gc.epoch, a.status, a.budget_ns);
    // every thread loads its share of all four partial arrays, then one tree
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = 0.0;
    for (int i = threadIdx.x; i < G; i += NT)
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] += __ldcg(a.partials + (slot + k) * G + i);
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; k++) s_w4[w][k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double c = 0.0;
        for (int i = 0; i < NT / 32; i++) c += s_w4[i][k];
        o[k] = c;
    }
}

__device__ __forceinline__ void grid_sync(const CgArgs &a, GridCtx &gc)
{
    gc.epoch++;
    gc.ok = gc.ok && MF_GRID_BARRIER(a.bar, gc.epoch, a.status, a.budget_ns);
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
        // CTA-wide vote on the bounded wait so that every thread leaves together
        if (!__syncthreads_and(mbar_wait_bounded(&S.bar[k], (gc.par >> (k)) & 1u, a.status, a.budget_ns))) {
            ok = false;
            // this stage and the other may still have copies in flight: wait
            // for them before leaving so no copy lands in freed memory
            mbar_drain(&S.bar[k], (gc.par >> (k)) & 1u, a.status, a.budget_ns);
            gc.par ^= 1u << (k);
            if (c + 1 < ce) {
                mbar_drain(&S.bar[k ^ 1], (gc.par >> (k ^ 1)) & 1u, a.status, a.budget_ns);
                gc.par ^= 1u << (k ^ 1);
            }
            break;
        }
        gc.par ^= 1u << (k);
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

// One row from the row-slot layout.  mt, vd / hd point at the row's first
// slot word / value / slot header; consecutive slots are MF_TILE elements
// (words, values) or one header apart.  pay + (header >> 2) * 16 is a slot's
// payload.  FP64 (PK 0): per-tile partial sums in the reference's order,
// products and sums rounded separately (bit-identical to blockspmv_cpu);
// mixed (PK 1): the slot's format decoded to FP32, fused multiply-add
// accumulation in row order.  U slots are loaded before any is used.
template <int PK, class Src>
__device__ __forceinline__ double slot_row(const unsigned short *mt, const double *vd, const unsigned *hd,
                                           const unsigned char *pay, const int *tcol, int K, int row, int hl, Src src,
                                           double &xown, bool &has_own)
{
    using XT = decltype(src(0));
    constexpr int U = SLOT_U;
    double yd = 0.0, part = 0.0;
    float yf = 0.f;
    int prevj = -1;
    has_own = false;
    for (int kk = 0; kk < K; kk += U) {
        unsigned short m[U];
        double v[U];
        float f[U];
        int col[U];
        XT xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = kk + u;
            const bool in = k < K;
            m[u] = in ? mt[k * MF_TILE] : (unsigned short)0xFFFF;
            if constexpr (PK == 0) {
                v[u] = in ? vd[k * MF_TILE] : 0.0;
            } else {
                f[u] = 0.f;
                if (in) {
                    const unsigned h = hd[k];
                    const unsigned char *d = pay + (size_t)(h >> 2) * 16;
                    const unsigned fm = h & 3u;
                    if (fm == 0u) f[u] = ((const float *)d)[hl];
                    else if (fm == 1u) f[u] = __half2float(((const __half *)d)[hl]);
                    else if (fm == 2u) f[u] = (float)((const signed char *)d)[hl];
                    else m[u] = 0xFFFF;  // every tile of this slot is bypassed
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) col[u] = (m[u] != 0xFFFF) ? tcol[m[u] >> 4] * MF_TILE + (m[u] & 15) : -1;
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = (col[u] >= 0) ? src(col[u]) : (XT)0;
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (col[u] < 0) continue;
            if (col[u] == row) {
                xown = (double)xv[u];
                has_own = true;
            }
            if constexpr (PK == 0) {
                const int j = m[u] >> 4;
                if (j != prevj) {
                    yd = __dadd_rn(yd, part);
                    part = 0.0;
                    prevj = j;
                }
                part = __dadd_rn(part, __dmul_rn((double)xv[u], v[u]));
            } else {
                yf = fmaf(f[u], (float)xv[u], yf);
            }
        }
    }
    if constexpr (PK == 0) return __dadd_rn(yd, part);
    else return (double)yf;
}

__device__ __forceinline__ SlotChunk slot_rec(const CgArgs &a, const SlotSmem &S, int cb, int c)
{
    return (c - cb < SRECS) ? S.recs[c - cb] : a.schunks[c];
}

// Thread 0: stage slot chunk c into stage k.
template <int PK>
__device__ void issue_slot_chunk(const CgArgs &a, SlotSmem &S, int c, int k)
{
    const int cb = a.scta_chunk[blockIdx.x];
    const SlotChunk r = slot_rec(a, S, cb, c);
    SlotHdr &h = S.hdr[k];
    h.rec = r;
    unsigned char *st = S.stage[k];
    const long long m0 = 2ll * MF_TILE * r.k0, m1 = 2ll * MF_TILE * r.k1;
    unsigned total = range_bytes(4ll * r.s0, 4ll * (r.s1 + 1)) * 2;
    if (!r.direct) {
        total += range_bytes(4ll * r.t0, 4ll * r.t1) + range_bytes(m0, m1);
        if (PK == 0) total += range_bytes(8ll * MF_TILE * r.k0, 8ll * MF_TILE * r.k1);
        else total += range_bytes(4ll * r.k0, 4ll * (r.k1 + 1)) + range_bytes(r.y0, r.y1);
    }
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.bar[k], total);
    add_range(st + SOFF_SSLOT, (const unsigned char *)a.sslot, 4ll * r.s0, 4ll * (r.s1 + 1), &S.bar[k], h.sh_sslot);
    add_range(st + SOFF_TPTR, (const unsigned char *)a.A.tile_ptr, 4ll * r.s0, 4ll * (r.s1 + 1), &S.bar[k],
              h.sh_tptr);
    if (r.direct) return;
    add_range(st + SOFF_TCOL, (const unsigned char *)a.A.tile_columnidx, 4ll * r.t0, 4ll * r.t1, &S.bar[k],
              h.sh_tcol);
    add_range(st + SOFF_META, (const unsigned char *)a.smeta, m0, m1, &S.bar[k], h.sh_meta);
    if (PK == 0) {
        add_range(st + SOFF_DATA, (const unsigned char *)a.sval, 8ll * MF_TILE * r.k0, 8ll * MF_TILE * r.k1, &S.bar[k],
                  h.sh_data);
    } else {
        add_range(st + SOFF_DATA, (const unsigned char *)a.shdr, 4ll * r.k0, 4ll * (r.k1 + 1), &S.bar[k], h.sh_data);
        add_range(st + SOFF_PAY, a.spay, r.y0, r.y1, &S.bar[k], h.sh_pay);
    }
}

// y = A src over this CTA's slot chunks [cb, ce); out(s, r, y, xown,
// has_own) receives every row.  Chunks stream through NSTG shared-memory
// stages: while the CTA computes one chunk (one half-warp per strip, one
// lane per row), the bulk copies of the next ones are landing; a stage is
// refilled as soon as the CTA is done with it.  Every thread waits for its
// chunk's data itself; a thread whose bounded wait expired computes nothing,
// and the barrier closing the chunk votes, so that the whole CTA leaves
// together -- after waiting (bounded) for the copies still in flight, so
// that none lands in freed shared memory.  Returns false when a wait expired.
template <int PK, class Src, class Out>
__device__ bool spmv_slots(const CgArgs &a, SlotSmem &S, GridCtx &gc, int cb, int ce, Src src, Out &out,
                           unsigned long long *tph)
{
    // optional thread-0 timers: [5] waiting for staged chunks, [6] computing
    // rows, [7] the closing barrier and the refill
    const bool timed = tph != nullptr && threadIdx.x == 0;
    unsigned long long tm = timed ? globaltimer_ns() : 0ull;
#define MF_SSUB(k)                                       \
    if (timed) {                                         \
        const unsigned long long nw_ = globaltimer_ns(); \
        tph[(k)] += nw_ - tm;                            \
        tm = nw_;                                        \
    }
    const MfTiles &A = a.A;
    const int tid = threadIdx.x, hw = tid >> 4, hl = tid & 15;
    if (tid == 0)
        for (int j = 0; j < NSTG && cb + j < ce; j++) issue_slot_chunk<PK>(a, S, cb + j, j);
    __syncthreads();
    for (int c = cb; c < ce; c++) {
        const int k = (c - cb) % NSTG;
        const bool w = mbar_wait_bounded(&S.bar[k], (gc.par >> (k)) & 1u, a.status, a.budget_ns);
        gc.par ^= 1u << (k);
        MF_SSUB(5);
        const SlotHdr &h = S.hdr[k];
        const SlotChunk &rec = h.rec;
        // the header is valid whether or not the data arrived (written before
        // the copies were issued), so L and the barriers below are uniform
        const int L = rec.lanes;
        if (L == 1) {
            // one half-warp per strip, one lane per row, from the stage
            const int s = rec.s0 + hw;
            if (w && s < rec.s1) {
                const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
                if (hl < rowlen) {
                    const unsigned char *st = S.stage[k];
                    const int *ssl = (const int *)(st + SOFF_SSLOT + h.sh_sslot);
                    const int *tpt = (const int *)(st + SOFF_TPTR + h.sh_tptr);
                    const int kA = ssl[hw] - rec.k0, K = ssl[hw + 1] - ssl[hw];
                    const unsigned short *mt =
                        (const unsigned short *)(st + SOFF_META + h.sh_meta) + kA * MF_TILE + hl;
                    const double *vd = (const double *)(st + SOFF_DATA + h.sh_data) + kA * MF_TILE + hl;
                    const unsigned *hd = (const unsigned *)(st + SOFF_DATA + h.sh_data) + kA;
                    const unsigned char *pay = st + SOFF_PAY + h.sh_pay - rec.y0;
                    const int *tcl = (const int *)(st + SOFF_TCOL + h.sh_tcol) + (tpt[hw] - rec.t0);
                    double xown = 0.0;
                    bool own = false;
                    const double y = slot_row<PK>(mt, vd, hd, pay, tcl, K, s * MF_TILE + hl, hl, src, xown, own);
                    out(s, hl, y, xown, own);
                }
            }
        } else {
            // L half-warps per strip, each on a contiguous part of its slots;
            // the parts' sums are added in order
            const int j = hw / L, part = hw % L;
            const int s = rec.s0 + j;
            const bool row_ok = w && s < rec.s1 && hl < ((s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE);
            double y = 0.0, xown = 0.0;
            bool own = false;
            if (row_ok) {
                const unsigned char *st = S.stage[k];
                const int *ssl = (const int *)(st + SOFF_SSLOT + h.sh_sslot);
                const int *tpt = (const int *)(st + SOFF_TPTR + h.sh_tptr);
                const int K = ssl[j + 1] - ssl[j];
                const int kb = K * part / L, ke = K * (part + 1) / L;
                const int row = s * MF_TILE + hl;
                if (rec.direct) {
                    // one strip too large for a stage: read from global memory
                    const int k0 = ssl[0] + kb;
                    const size_t e0 = (size_t)k0 * MF_TILE + hl;
                    y = slot_row<PK>(a.smeta + e0, a.sval + e0, a.shdr + k0, a.spay, A.tile_columnidx + tpt[0],
                                     ke - kb, row, hl, src, xown, own);
                } else {
                    const int kA = ssl[j] - rec.k0 + kb;
                    const unsigned short *mt =
                        (const unsigned short *)(st + SOFF_META + h.sh_meta) + kA * MF_TILE + hl;
                    const double *vd = (const double *)(st + SOFF_DATA + h.sh_data) + kA * MF_TILE + hl;
                    const unsigned *hd = (const unsigned *)(st + SOFF_DATA + h.sh_data) + kA;
                    const unsigned char *pay = st + SOFF_PAY + h.sh_pay - rec.y0;
                    const int *tcl = (const int *)(st + SOFF_TCOL + h.sh_tcol) + (tpt[j] - rec.t0);
                    y = slot_row<PK>(mt, vd, hd, pay, tcl, ke - kb, row, hl, src, xown, own);
                }
            }
            S.py[tid] = y;
            S.px[tid] = xown;
            S.pown[tid] = own ? 1 : 0;
            __syncthreads();
            if (row_ok && part == 0) {
                double yy = 0.0, xo = 0.0;
                bool ow = false;
                for (int q = 0; q < L; q++) {
                    const int t = ((j * L + q) << 4) | hl;
                    yy = __dadd_rn(yy, S.py[t]);
                    if (!ow && S.pown[t]) {
                        ow = true;
                        xo = S.px[t];
                    }
                }
                out(s, hl, yy, xo, ow);
            }
        }
        MF_SSUB(6);
        if (!__syncthreads_and(w)) {
            // chunks c .. c+NSTG-1 may still be landing
            mbar_drain(&S.bar[k], ((gc.par >> k) & 1u) ^ 1u, a.status, a.budget_ns);
            for (int jj = 1; jj < NSTG && c + jj < ce; jj++) {
                const int kj = (c + jj - cb) % NSTG;
                mbar_drain(&S.bar[kj], (gc.par >> (kj)) & 1u, a.status, a.budget_ns);
                gc.par ^= 1u << (kj);
            }
            __syncthreads();
            return false;
        }
        if (tid == 0 && c + NSTG < ce) issue_slot_chunk<PK>(a, S, c + NSTG, k);
        MF_SSUB(7);
    }
#undef MF_SSUB
    return true;
}

// ---- staged slot chunks ----
//
// Stage layout: strip descriptors, slot positions, FP64 values or the mixed
// slot headers and payload, then the staged vectors (the chunk's column runs
// of one FP64 vector or of two vectors of the solver's type, one after the
// other, SC_XCAP elements apart).  Every region is 16-byte aligned and sized
// for the largest 16-byte-rounded range it receives.
template <bool MIX>
struct StagedCfg {
    static constexpr int OFF_SDESC = 0;  // strip descriptors (8 bytes each)
    static constexpr int OFF_META = (SC_STRIPS * 8 + 32 + 15) / 16 * 16;
    static constexpr int OFF_DATA = OFF_META + SC_SLOTS * MF_TILE * 2 + 32;
    static constexpr int OFF_PAY = OFF_DATA + SC_SLOTS * 4 + 32;
    static constexpr int OFF_VEC = MIX ? OFF_PAY + SC_SLOTS * 64 + 32 : OFF_DATA + SC_SLOTS * MF_TILE * 8 + 32;
    static constexpr int VEC_BYTES = SC_XCAP * 8 * (MIX ? 1 : 2);
    static constexpr int STAGE = OFF_VEC + VEC_BYTES;
    static_assert(OFF_META % 16 == 0 && OFF_DATA % 16 == 0 && OFF_PAY % 16 == 0 && OFF_VEC % 16 == 0 &&
                      STAGE % 16 == 0 && SC_XCAP % 16 == 0,
                  "staged regions must be 16-byte aligned");
};
#ifndef MF_STAGED_RECS
#define MF_STAGED_RECS 32
#endif
constexpr int TRECS = MF_STAGED_RECS;  // staged chunk records cached in shared memory

template <bool MIX>
struct __align__(16) StagedSmem {
    unsigned char stage[NSTG][StagedCfg<MIX>::STAGE];
    SlotHdr hdr[NSTG];
    SlotChunk recs[TRECS];
    double py[NT], px[NT];
    unsigned char pown[NT];
    uint64_t bar[NSTG];
    double warp[NT / 32];
    double res;
};

// The first STAGED_ARRIVALS warps (all their lanes) stage chunk c into
// stage k.  With 2 warps, warp 0 copies the chunk record into the stage
// header and issues the range copies (range 0 strip descriptors, 1 slot
// positions, 2 the values (PK 0) or mixed headers (PK 1) when STV, 3 the
// mixed payload when STV; lane i issues range i) and warp 1 the chunk's
// column runs (lane j < nrun: run j of v0, nrun <= j < 2 nrun when NV is 2:
// run j - nrun of v1).  With 4 warps, warp 0 takes the record and ranges 0-1,
// warp 1 ranges 2-3, warp 2 the runs of v0 and warp 3 those of v1.  Each
// warp sums its bytes across its lanes and its lane 0 arrives on the stage's
// mbarrier with them as expected transactions before the warp issues a copy,
// so the phase (one arrival per warp) completes only when every warp's
// copies have landed.  The caller has fenced the vectors (see spmv_staged).
#ifndef MF_STAGED_ISSUE_WARPS
#define MF_STAGED_ISSUE_WARPS 4
#endif
constexpr int STAGED_ARRIVALS = MF_STAGED_ISSUE_WARPS;
static_assert(STAGED_ARRIVALS == 2 || STAGED_ARRIVALS == 4, "the refill runs on 2 or 4 warps");
template <int PK, bool STV, typename VT, int NV, bool MIX>
__device__ __forceinline__ void issue_staged(const CgArgs &a, StagedSmem<MIX> &S, int cb, int c, int k, const VT *v0,
                                             const VT *v1)
{
    using C = StagedCfg<MIX>;
    static_assert(NV * SC_RUNS <= 32, "one run copy per lane");
    constexpr int RW = (int)(sizeof(SlotChunk) / 4);
    static_assert(sizeof(SlotChunk) % 4 == 0 && RW <= 32, "the record is copied one word per lane");
    constexpr int W = STAGED_ARRIVALS;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const bool runs = W == 2 ? wp == 1 : wp >= 2;
    const SlotChunk *src = c - cb < TRECS ? &S.recs[c - cb] : &a.schunks[c];
    unsigned char *st = S.stage[k];
    const unsigned char *g = nullptr;
    unsigned char *d = nullptr;
    unsigned bytes = 0;
    if (!runs) {
        SlotHdr &h = S.hdr[k];
        if (wp == 0 && lane < RW) ((int *)&h.rec)[lane] = ((const int *)src)[lane];
        const int rid = W == 2 ? lane : wp == 0 ? (lane < 2 ? lane : 4) : lane + 2;  // the range of this lane
        long long a0 = 0, a1 = 0;
        int *shift = nullptr;
        if (rid == 0) {
            g = (const unsigned char *)a.sdesc, d = st + C::OFF_SDESC, a0 = 8ll * src->s0, a1 = 8ll * src->s1;
            shift = &h.sh_sslot;
        } else if (rid == 1) {
            g = (const unsigned char *)a.spos, d = st + C::OFF_META;
            a0 = 2ll * MF_TILE * src->k0, a1 = 2ll * MF_TILE * src->k1;
            shift = &h.sh_meta;
        } else if (rid == 2 && STV) {
            d = st + C::OFF_DATA;
            shift = &h.sh_data;
            if (PK == 0) g = (const unsigned char *)a.sval, a0 = 8ll * MF_TILE * src->k0, a1 = 8ll * MF_TILE * src->k1;
            else g = (const unsigned char *)a.shdr, a0 = 4ll * src->k0, a1 = 4ll * (src->k1 + 1);
        } else if (rid == 3 && STV && PK == 1) {
            g = a.spay, d = st + C::OFF_PAY, a0 = src->y0, a1 = src->y1;
            shift = &h.sh_pay;
        }
        // whole 16-byte words around [a0, a1); the shift locates a0
        if (shift) {
            const long long c0 = a0 & ~15ll, c1 = (a1 + 15) & ~15ll;
            *shift = (int)(a0 - c0);
            g += c0;
            bytes = (unsigned)(c1 - c0);
        }
    } else {
        const int nrun = src->nrun;
        // copy q: run q of v0 (q < nrun) or run q - nrun of v1
        const int q = W == 2 ? lane : wp == 3 ? lane + nrun : lane;
        if (W == 2 ? lane < NV * nrun : lane < nrun && (wp == 2 || NV == 2)) {
            const bool second = q >= nrun;
            const int j = second ? q - nrun : q;
            g = (const unsigned char *)((second ? v1 : v0) + src->rg[j]);
            d = st + C::OFF_VEC + (size_t)((second ? SC_XCAP : 0) + src->rs[j]) * sizeof(VT);
            bytes = (unsigned)src->rl[j] * (unsigned)sizeof(VT);
        }
    }
    unsigned total = bytes;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
    fence_proxy_async_smem();
    if (lane == 0) {
        if (total) mbar_arrive_expect_tx(&S.bar[k], total);
        else mbar_arrive(&S.bar[k]);  // nothing to copy for this warp
    }
    __syncwarp();
    if (bytes) {
        if (!runs) bulk_g2s_hint(d, g, bytes, &S.bar[k], l2_policy_evict_first());
        else bulk_g2s(d, g, bytes, &S.bar[k]);
    }
}

// One row from a staged chunk: the slot words are positions in the staged
// vectors, whose entry is v0 (NV 1) or bt * v1 + v0 (NV 2, one rounding);
// otherwise as slot_row (the position's tile, pos >> 4, changes exactly
// where the tile column does, so the FP64 per-tile partial sums are those of
// blockspmv_cpu).  vd may point to shared or global memory.
#ifndef MF_STAGED_UNROLL
#define MF_STAGED_UNROLL 8
#endif
constexpr int STAGED_UNROLL = MF_STAGED_UNROLL;

__device__ __forceinline__ float fma_vt(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_vt(double a, double b, double c) { return fma(a, b, c); }

// One FP64 row from a staged chunk: the slot words are positions in the
// staged vectors, whose entry is v0 (NV 1) or bt * v1 + v0 (NV 2, one
// rounding); per-tile partial sums as slot_row (the position's tile, pos >>
// 4, changes exactly where the tile column does, so the sums round as
// blockspmv_cpu's).  vd may point to shared or global memory.
template <int NV>
__device__ __forceinline__ double staged_row_fp64(const unsigned short *mt, const double *vd, int K, const double *sv0,
                                                  const double *sv1, double bt)
{
    double yd = 0.0, part = 0.0;
    int prevj = -1;
#pragma unroll STAGED_UNROLL
    for (int k = 0; k < K; k++) {
        const unsigned m = mt[k * MF_TILE];
        const double v = vd[k * MF_TILE];
        if (m == 0xFFFFu) continue;
        const double xv = NV == 2 ? fma(bt, sv1[m], sv0[m]) : sv0[m];
        const int j = (int)(m >> 4);
        if (j != prevj) {
            yd = __dadd_rn(yd, part);
            part = 0.0;
            prevj = j;
        }
        part = __dadd_rn(part, __dmul_rn(xv, v));
    }
    return __dadd_rn(yd, part);
}

// One mixed row from a staged chunk: FP32 fused multiply-add accumulation in
// row order of v = bt * v1 + v0 times the slot value decoded to FP32, empty
// entries and bypassed slots skipped (the same operations as slot_row).
// FMT 0 / 1 / 2: every slot of the chunk is fp32 / fp16 / int8, so slot k's
// 16 values sit at pay_u + k * (64 >> FMT); FMT -1: each slot's header gives
// its format and payload offset.  No branches: a skipped entry reads a
// valid position and leaves the sum unchanged.
template <int FMT>
__device__ __forceinline__ float staged_row_mixed(const unsigned short *mt, const unsigned *hd, const unsigned char *pay,
                                                  const unsigned char *pay_u, int K, int hl, const float *sv0,
                                                  const float *sv1, float bt)
{
    float yf = 0.f;
#pragma unroll STAGED_UNROLL
    for (int k = 0; k < K; k++) {
        const unsigned m = mt[k * MF_TILE];
        float f;
        bool use = m != 0xFFFFu;
        if constexpr (FMT == 0) {
            f = ((const float *)(pay_u + k * 64))[hl];
        } else if constexpr (FMT == 1) {
            f = __half2float(((const __half *)(pay_u + k * 32))[hl]);
        } else if constexpr (FMT == 2) {
            f = (float)((const signed char *)(pay_u + k * 16))[hl];
        } else {
            const unsigned h = hd[k];
            const unsigned char *d = pay + (h >> 2) * 16u;
            const unsigned fm = h & 3u;
            if (fm == 0u) f = ((const float *)d)[hl];
            else if (fm == 1u) f = __half2float(((const __half *)d)[hl]);
            else f = (float)((const signed char *)d)[hl];
            use = use && fm != 3u;  // every tile of this slot is bypassed
        }
        const unsigned mm = use ? m : 0u;
        const float xv = fmaf(bt, sv1[mm], sv0[mm]);
        yf = use ? fmaf(f, xv, yf) : yf;
    }
    return yf;
}

// y = A v over this CTA's staged chunks [cb, ce), v = v0 (NV 1) or
// bt * v1 + v0 (NV 2); out(s, r, y, xown, has_own) receives every row, xown
// being the row's own entry of v when its column is staged.  No row reads a
// vector from global memory.  STV false leaves the values in global memory
// (a.sval: the FP64 refinement SpMV of the mixed kernel, whose stages are
// sized for the mixed payload).
//
// Only thread 0 waits on the stage barriers: after computing chunk c it
// waits (bounded) for chunk c+1, and the CTA barrier that closes chunk c
// hands the result to every thread, which then reads chunk c+1's stage (the
// copies' writes, observed by thread 0 through the mbarrier, are ordered
// before the other threads' reads by that barrier).  One CTA barrier per
// chunk, and no warp sleeps in an mbarrier wait.  The barrier votes: when a
// wait expired, the copies still in flight are drained (bounded, at least
// one second) before the CTA leaves, so none lands in freed shared memory.
// Optional thread-0 timers: [5] waiting for the next chunk, [6] computing
// rows, [7] the closing barrier and the refill.
template <int PK, bool STV, typename VT, int NV, bool MIX, class Out>
__device__ bool spmv_staged(const CgArgs &a, StagedSmem<MIX> &S, GridCtx &gc, int cb, int ce, const VT *v0,
                            const VT *v1, VT bt, Out &out, unsigned long long *tph)
{
    using C = StagedCfg<MIX>;
    static_assert(NV * SC_XCAP * (int)sizeof(VT) <= C::VEC_BYTES, "staged vectors must fit the stage");
    static_assert(STV || PK == 0, "mixed payload is always staged");
    static_assert(!STV || PK == 1 || !MIX, "FP64 values are staged only in FP64 stages");
    const bool timed = tph != nullptr && threadIdx.x == 0;
    unsigned long long tm = timed ? globaltimer_ns() : 0ull;
#define MF_TSUB(k)                                       \
    if (timed) {                                         \
        const unsigned long long nw_ = globaltimer_ns(); \
        tph[(k)] += nw_ - tm;                            \
        tm = nw_;                                        \
    }
    const MfTiles &A = a.A;
    const int tid = threadIdx.x, hw = tid >> 4, hl = tid & 15;
    if (tid < 32 * STAGED_ARRIVALS) {
        // the vectors were written earlier in this kernel by ordinary stores
        // of other CTAs, made visible here by the grid barrier; the proxy
        // fence orders them before the bulk copies, which read through the
        // async proxy.  They do not change during the pass.
        asm volatile("fence.proxy.async.global;\n" ::: "memory");
        for (int j = 0; j < NSTG && cb + j < ce; j++) issue_staged<PK, STV, VT, NV>(a, S, cb, cb + j, j, v0, v1);
    }
    // copies of chunks [c0, c0 + n) may be in flight: wait for them
    // (bounded) before leaving, each with the parity its stage expects
    auto drain = [&](int c0, int n) {
        for (int jj = 0; jj < n && c0 + jj < ce; jj++) {
            const int kj = (c0 + jj - cb) % NSTG;
            if (tid == 0) mbar_drain(&S.bar[kj], (gc.par >> kj) & 1u, a.status, a.budget_ns);
            gc.par ^= 1u << kj;
        }
        __syncthreads();
    };
    {
        bool w0 = true;
        if (tid == 0 && cb < ce) w0 = mbar_wait_bounded(&S.bar[0], gc.par & 1u, a.status, a.budget_ns);
        if (!__syncthreads_and(w0)) {
            drain(cb, NSTG);  // the chunks issued so far
            return false;
        }
        if (cb < ce) gc.par ^= 1u;
    }
    for (int c = cb; c < ce; c++) {
        const int k = (c - cb) % NSTG;
        const SlotHdr &h = S.hdr[k];
        const SlotChunk &rec = h.rec;
        const int L = rec.lanes;
        const int j = L == 1 ? hw : hw / L, part = L == 1 ? 0 : hw % L;
        const int s = rec.s0 + j;
        const bool row_ok = s < rec.s1 && hl < ((s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE);
        // FP32 sums stay FP32 until the caller converts them (mixed payload)
        using YT = typename std::conditional<PK == 0, double, float>::type;
        YT y = 0;
        VT xown = 0;
        bool own = false;
        if (row_ok) {
            const unsigned char *st = S.stage[k];
            // one load: the strip's first slot in the chunk, its slot count
            // and the offset from a row to its own staged position
            const int2 dsc = ((const int2 *)(st + C::OFF_SDESC + h.sh_sslot))[j];
            const int K = dsc.x >> 16;
            const int kb = L == 1 ? 0 : K * part / L, ke = L == 1 ? K : K * (part + 1) / L;
            const int row = s * MF_TILE + hl;
            const int ownpos = dsc.y == INT_MIN ? -1 : row + dsc.y;
            const int kA = (dsc.x & 0xFFFF) + kb;
            const unsigned short *mt = (const unsigned short *)(st + C::OFF_META + h.sh_meta) + kA * MF_TILE + hl;
            const VT *sv0 = (const VT *)(st + C::OFF_VEC), *sv1 = sv0 + SC_XCAP;
            if constexpr (PK == 0) {
                const double *vd = STV ? (const double *)(st + C::OFF_DATA + h.sh_data) + kA * MF_TILE + hl
                                       : a.sval + (size_t)(rec.k0 + kA) * MF_TILE + hl;
                y = staged_row_fp64<NV>(mt, vd, ke - kb, (const double *)sv0, (const double *)sv1, (double)bt);
            } else {
                const unsigned *hd = (const unsigned *)(st + C::OFF_DATA + h.sh_data) + kA;
                const unsigned char *pay = st + C::OFF_PAY + h.sh_pay - rec.y0;
                const unsigned char *pay0 = st + C::OFF_PAY + h.sh_pay;  // first slot of the chunk
                const float *f0 = (const float *)sv0, *f1 = (const float *)sv1;
                const float fb = (float)bt;
                if (rec.fmt == 0) y = staged_row_mixed<0>(mt, hd, pay, pay0 + kA * 64, ke - kb, hl, f0, f1, fb);
                else if (rec.fmt == 1) y = staged_row_mixed<1>(mt, hd, pay, pay0 + kA * 32, ke - kb, hl, f0, f1, fb);
                else if (rec.fmt == 2) y = staged_row_mixed<2>(mt, hd, pay, pay0 + kA * 16, ke - kb, hl, f0, f1, fb);
                else y = staged_row_mixed<-1>(mt, hd, pay, pay0, ke - kb, hl, f0, f1, fb);
            }
            // the row's own entry of v (its column is staged when the chunk
            // holds its diagonal tile)
            if (ownpos >= 0) {
                if constexpr (NV == 2) xown = fma_vt(bt, sv1[ownpos], sv0[ownpos]);
                else xown = sv0[ownpos];
                own = true;
            }
        }
        if (L == 1) {
            if (row_ok) out(s, hl, y, xown, own);
        } else {
            // the parts' sums are added in order
            S.py[tid] = (double)y;
            S.px[tid] = (double)xown;
            S.pown[tid] = own ? 1 : 0;
            __syncthreads();
            if (row_ok && part == 0) {
                double yy = 0.0, xo = 0.0;
                bool ow = false;
                for (int q = 0; q < L; q++) {
                    const int t = ((j * L + q) << 4) | hl;
                    yy = __dadd_rn(yy, S.py[t]);
                    if (!ow && S.pown[t]) {
                        ow = true;
                        xo = S.px[t];
                    }
                }
                out(s, hl, yy, xo, ow);
            }
        }
        MF_TSUB(6);
        const int kn = (c + 1 - cb) % NSTG;
        bool wn = true;
        if (tid == 0 && c + 1 < ce) wn = mbar_wait_bounded(&S.bar[kn], (gc.par >> kn) & 1u, a.status, a.budget_ns);
        MF_TSUB(5);
        if (!__syncthreads_and(wn)) {
            drain(c + 1, NSTG - 1);  // chunks c+1 .. c+NSTG-1 (c+NSTG is not issued yet)
            return false;
        }
        if (c + 1 < ce) gc.par ^= 1u << kn;
        // every thread is done with stage k
        if (tid < 32 * STAGED_ARRIVALS && c + NSTG < ce) issue_staged<PK, STV, VT, NV>(a, S, cb, c + NSTG, k, v0, v1);
        MF_TSUB(7);
    }
#undef MF_TSUB
    return true;
}

// The SpMV of the layout the kernel was built for (LAY 0: staged tile
// chunks, LAY 1: row slots).
template <int PK, int LAY, class SM, class Src, class Out>
__device__ __forceinline__ bool spmv_any(const CgArgs &a, SM &S, GridCtx &gc, int cb, int ce, int sb, int se,
                                         Src src, Out &out, unsigned long long *tph)
{
    if constexpr (LAY == 0) {
        return spmv_chunks<PK>(a, S, gc, cb, ce, src, out, tph);
    } else {
        return spmv_slots<PK>(a, S, gc, cb, ce, src, out, tph);
    }
}

}  // namespace persist
}  // namespace mf
