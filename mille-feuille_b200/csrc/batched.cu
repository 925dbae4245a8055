// batched.cu -- many independent CG solves of uneven size in one launch.
//
// No reference counterpart: the reference solves one system per launch.
// Design for B200: the systems are sorted by size and handed out by a device
// work queue to thread-block clusters; a cluster of C CTAs solves one system
// at a time.  The system's rows are split across the cluster's CTAs, the
// SpMV reads the row-major execution layout of the system (entries of a row
// in the tile order of the reference format, which for the random systems of
// this workload is column order), several lanes per row, and every dot
// product is reduced through distributed shared memory with a hardware
// cluster barrier -- no grid-wide synchronisation, so small systems cost no
// more than their own iterations.  Each cluster keeps iterating until its
// system reaches the tolerance, then takes the next system.  Mixed policy:
// FP32 values and vectors, FP32 accumulation, FP64 dot products, and FP64
// reliable updates from the FP64 values, as in the single-system solver.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include <type_traits>

#include "mf_internal.h"
#include "tma.cuh"

namespace cg = cooperative_groups;

struct mf_batch_s {
    int count = 0;
    long long rows_total = 0, nnz_total = 0;
    std::vector<int> n;           // rows per system (caller order)
    std::vector<long long> row0;  // first row of each system (caller order)
    int *d_order = nullptr;       // systems by descending size
    long long *d_row0 = nullptr, *d_nz0 = nullptr;
    int *d_n = nullptr;
    int *d_rowptr = nullptr;      // per system, relative to the system's first entry
    int *d_col = nullptr;
    double *d_val = nullptr;
    float *d_val32 = nullptr;
    // per-system results
    int *d_iters = nullptr, *d_refs = nullptr, *d_status = nullptr;
    double *d_relres = nullptr;
    void *work = nullptr;
    size_t work_bytes = 0;
    int *d_queue = nullptr;
    // row chunks of every system (staged through shared memory by the SpMV)
    int *d_sc = nullptr;          // [count+1] first chunk of each system
    int *d_crow = nullptr;        // per system nch+1 chunk row starts (relative rows), at sc[s] + s
    int *d_cent = nullptr;        // the entries offsets rowptr[crow] of the same chunks
    // CUDA graph of the last solve configuration
    cudaGraphExec_t graph = nullptr;
    const void *graph_b = nullptr;
    void *graph_x = nullptr;
    int graph_key[6] = {0, 0, 0, 0, 0, 0};
    int tuned_lanes = 0, tuned_cluster = 0;
};

namespace mf {
namespace {

constexpr int BNT = 256;

struct BatchArgs {
    int count;
    const int *order;
    const int *n;
    const long long *row0, *nz0;
    const int *rowptr, *col;
    const double *val;
    const float *val32;
    const double *b;
    double *x;
    void *r, *p0, *p1, *q, *xlo;  // workspace vectors (rows_total each)
    const int *sc, *crow, *cent;   // row chunks
    int *queue;
    int *iters, *refs, *status;
    double *relres;
    int maxiter;
    double tol;
    double delta;
    unsigned long long budget_ns;  // bound of every shared-memory stage wait
};

// Deterministic cluster-wide sum: each CTA reduces its threads in a fixed
// tree, publishes the value in its shared memory, and after the cluster
// barrier every CTA adds the CTAs' values in rank order.
__device__ __forceinline__ double cluster_sum(cg::cluster_group &cl, double v, double *slot, double *s_warp)
{
    const double c = block_sum<BNT>(v, s_warp);
    if (threadIdx.x == 0) *slot = c;
    cl.sync();
    double s = 0.0;
    const unsigned ncta = cl.num_blocks();
    for (unsigned k = 0; k < ncta; k++) s += *cl.map_shared_rank(slot, k);
    return s;
}

// Row chunks staged through shared memory: up to BCR rows and BCE entries
// per chunk (a longer row is a chunk of its own, read from global memory).
constexpr int BCE = 2048, BCR = 256;
constexpr int BOFF_RP = 0;                          // rowptr[r0 .. r1]
constexpr int BOFF_COL = 1072;                      // columns of the chunk's entries
constexpr int BOFF_VAL = BOFF_COL + BCE * 4 + 32;   // values (FP64, or FP32 when mixed)
constexpr int BSTAGE = BOFF_VAL + BCE * 8 + 32;
static_assert(BOFF_COL % 16 == 0 && BOFF_VAL % 16 == 0 && BSTAGE % 16 == 0, "stage regions 16-byte aligned");
static_assert((BCR + 1) * 4 + 32 <= BOFF_COL, "row pointers fit");

struct BHdr {
    int r0, r1, e0, direct;   // rows [r0, r1), first entry e0 (relative to the system)
    int sh_rp, sh_col, sh_val, pad;
};

#ifndef MF_BATCH_STAGES
#define MF_BATCH_STAGES 2
#endif
constexpr int BNS = MF_BATCH_STAGES;  // chunks in flight per CTA

struct BSmem {
    unsigned char stage[BNS][BSTAGE];
    BHdr hdr[BNS];
    uint64_t bar[BNS];
};

__device__ __forceinline__ void b_add_range(unsigned char *dst, const unsigned char *src, long long a0, long long a1,
                                            uint64_t *bar, int &shift)
{
    const long long c0 = a0 & ~15ll, c1 = (a1 + 15) & ~15ll;
    shift = (int)(a0 - c0);
    if (c1 > c0) bulk_g2s_hint(dst, src + c0, (unsigned)(c1 - c0), bar, l2_policy_evict_first());
}

__device__ __forceinline__ unsigned b_range_bytes(long long a0, long long a1)
{
    return (unsigned)(((a1 + 15) & ~15ll) - (a0 & ~15ll));
}

// A chunk's rows [r0, r1) and entries [e0, e1) (relative to its system).
struct BChunk {
    int r0, r1, e0, e1;
};

__device__ __forceinline__ BChunk b_chunk(const BatchArgs &a, int sys, int c)
{
    BChunk ch;
    ch.r0 = a.crow[c + sys];
    ch.r1 = a.crow[c + 1 + sys];
    ch.e0 = a.cent[c + sys];
    ch.e1 = a.cent[c + 1 + sys];
    return ch;
}

// Thread 0: stage chunk `ch` of system `sys` into stage k.
template <bool MIX>
__device__ void b_issue(const BatchArgs &a, BSmem &S, long long rp_base, long long z0, const BChunk &ch, int k)
{
    BHdr &h = S.hdr[k];
    const int r0 = ch.r0, r1 = ch.r1, e0 = ch.e0, e1 = ch.e1;
    h.r0 = r0;
    h.r1 = r1;
    h.e0 = e0;
    h.direct = (e1 - e0 > BCE) ? 1 : 0;
    const int vb = MIX ? 4 : 8;
    unsigned total = b_range_bytes(4 * (rp_base + r0), 4 * (rp_base + r1 + 1));
    if (!h.direct) total += b_range_bytes(4 * (z0 + e0), 4 * (z0 + e1)) + b_range_bytes(vb * (z0 + e0), vb * (z0 + e1));
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.bar[k], total);
    unsigned char *st = S.stage[k];
    b_add_range(st + BOFF_RP, (const unsigned char *)a.rowptr, 4 * (rp_base + r0), 4 * (rp_base + r1 + 1), &S.bar[k],
                h.sh_rp);
    if (h.direct) return;
    b_add_range(st + BOFF_COL, (const unsigned char *)a.col, 4 * (z0 + e0), 4 * (z0 + e1), &S.bar[k], h.sh_col);
    if (MIX)
        b_add_range(st + BOFF_VAL, (const unsigned char *)a.val32, 4 * (z0 + e0), 4 * (z0 + e1), &S.bar[k], h.sh_val);
    else
        b_add_range(st + BOFF_VAL, (const unsigned char *)a.val, 8 * (z0 + e0), 8 * (z0 + e1), &S.bar[k], h.sh_val);
}

// L lanes per row: lanes stride over the row's entries (BU entries per lane
// loaded before any is used); the partials are combined with a fixed xor
// tree, so every run gives the same bits.  Two rows per lane group are in
// flight at once (i1 < 0: none).
#ifndef MF_BATCH_BU
#define MF_BATCH_BU 8
#endif
constexpr int BU = MF_BATCH_BU;

// Row bounds of the two rows of a step (0, 0 for a missing row).
struct RowPair {
    int a0, e0, a1, e1;
};

__device__ __forceinline__ RowPair row_pair(const int *__restrict__ rp, int i0, int i1)
{
    RowPair p;
    p.a0 = (i0 >= 0) ? rp[i0] : 0;
    p.e0 = (i0 >= 0) ? rp[i0 + 1] : 0;
    p.a1 = (i1 >= 0) ? rp[i1] : 0;
    p.e1 = (i1 >= 0) ? rp[i1 + 1] : 0;
    return p;
}

template <int L, bool MIX, class Src, bool GLOBAL = true>
__device__ __forceinline__ void row_dot2(const RowPair &rb, const int *__restrict__ col,
                                         const double *__restrict__ val, const float *__restrict__ val32, int lane,
                                         Src src, double &y0, double &y1)
{
    using XT = decltype(src(0));
    const int a0 = rb.a0, e0 = rb.e0, a1 = rb.a1, e1 = rb.e1;
    double s0 = 0.0, s1 = 0.0;
    float f0 = 0.0f, f1 = 0.0f;
    const int n0 = e0 - a0, n1 = e1 - a1, nmax = n0 > n1 ? n0 : n1;
    for (int k = lane; k < nmax; k += L * BU) {
        int c0[BU], c1[BU];
        double v0[BU], v1[BU];
        float w0[BU], w1[BU];
#pragma unroll
        for (int u = 0; u < BU; u++) {
            const int kk = k + u * L;
            const bool in0 = kk < n0, in1 = kk < n1;
            if constexpr (GLOBAL) {
                c0[u] = in0 ? __ldcs(col + a0 + kk) : -1;
                c1[u] = in1 ? __ldcs(col + a1 + kk) : -1;
                if (MIX) {
                    w0[u] = in0 ? __ldcs(val32 + a0 + kk) : 0.0f;
                    w1[u] = in1 ? __ldcs(val32 + a1 + kk) : 0.0f;
                } else {
                    v0[u] = in0 ? __ldcs(val + a0 + kk) : 0.0;
                    v1[u] = in1 ? __ldcs(val + a1 + kk) : 0.0;
                }
            } else {  // staged in shared memory
                c0[u] = in0 ? col[a0 + kk] : -1;
                c1[u] = in1 ? col[a1 + kk] : -1;
                if (MIX) {
                    w0[u] = in0 ? val32[a0 + kk] : 0.0f;
                    w1[u] = in1 ? val32[a1 + kk] : 0.0f;
                } else {
                    v0[u] = in0 ? val[a0 + kk] : 0.0;
                    v1[u] = in1 ? val[a1 + kk] : 0.0;
                }
            }
        }
        XT x0[BU], x1[BU];
#pragma unroll
        for (int u = 0; u < BU; u++) {
            x0[u] = c0[u] >= 0 ? src(c0[u]) : (XT)0;
            x1[u] = c1[u] >= 0 ? src(c1[u]) : (XT)0;
        }
#pragma unroll
        for (int u = 0; u < BU; u++) {
            if (MIX) {
                f0 = fmaf(w0[u], (float)x0[u], f0);
                f1 = fmaf(w1[u], (float)x1[u], f1);
            } else {
                s0 = fma(v0[u], (double)x0[u], s0);
                s1 = fma(v1[u], (double)x1[u], s1);
            }
        }
    }
    if (MIX) {
        s0 = (double)f0;
        s1 = (double)f1;
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o, L);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o, L);
    }
    y0 = s0;
    y1 = s1;
}

#ifndef MF_BATCH_MINB
#define MF_BATCH_MINB 2
#endif

template <int L, bool MIX>
__global__ void __launch_bounds__(BNT, MF_BATCH_MINB) k_batched_cg(BatchArgs a)
{
    using VT = typename std::conditional<MIX, float, double>::type;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double s_warp[BNT / 32];
    __shared__ double s_slot[4];
    __shared__ int s_sys;
    __shared__ int s_fail;
    extern __shared__ __align__(16) unsigned char b_smem_raw[];
    BSmem &S = *reinterpret_cast<BSmem *>(b_smem_raw);
    if (threadIdx.x == 0) {
        for (int k = 0; k < BNS; k++) mbar_init(&S.bar[k], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned use[BNS];
#pragma unroll
    for (int k = 0; k < BNS; k++) use[k] = 0;
    const unsigned rank = cl.block_rank(), ncta = cl.num_blocks();
    const int tid = threadIdx.x;
    const int lane = tid % L, grp = tid / L;
    constexpr int GPB = BNT / L;  // row groups per CTA
    for (;;) {
        if (rank == 0 && tid == 0) s_sys = atomicAdd(a.queue, 1);
        cl.sync();
        const int qi = *cl.map_shared_rank(&s_sys, 0);
        cl.sync();  // every CTA has read the index before rank 0 writes the next
        if (qi >= a.count) break;
        const int sys = a.order[qi];
        const int n = a.n[sys];
        const long long r0 = a.row0[sys], z0 = a.nz0[sys];
        const int *rp = a.rowptr + r0 + sys;  // n+1 entries per system
        const int *col = a.col + z0;
        const double *val = a.val + z0;
        const float *val32 = a.val32 + z0;
        const double *b = a.b + r0;
        double *x = a.x + r0;
        VT *r = (VT *)a.r + r0, *q = (VT *)a.q + r0, *xlo = (VT *)a.xlo + r0;
        VT *pb[2] = {(VT *)a.p0 + r0, (VT *)a.p1 + r0};
        // this CTA's chunks and rows
        const int sc0 = a.sc[sys], nch = a.sc[sys + 1] - sc0;
        const int cl0 = sc0 + (int)((long long)nch * rank / ncta), cl1 = sc0 + (int)((long long)nch * (rank + 1) / ncta);
        const int ra = a.crow[cl0 + sys], rb = a.crow[cl1 + sys];
        const long long rp_base = r0 + sys;
        double lb = 0.0, lr = 0.0;
        for (int i = ra + tid; i < rb; i += BNT) {
            const double bv = b[i];
            const VT rv = (VT)bv;
            x[i] = 0.0;
            r[i] = rv;
            pb[0][i] = (VT)0;
            if (MIX) xlo[i] = (VT)0;
            lb += bv * bv;
            lr += (double)rv * (double)rv;
        }
        const double bb = cluster_sum(cl, lb, &s_slot[0], s_warp);
        double rho = MIX ? cluster_sum(cl, lr, &s_slot[1], s_warp) : bb;
        const double nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
        double beta = 0.0, rmax = sqrt(rho), relres = sqrt(rho) / nb;
        int it = 0, refs = 0, status = MF_OK;
        while (true) {
            if (sqrt(rho) <= a.tol * nb) break;
            if (it >= a.maxiter) {
                status = MF_ERR_NOT_CONVERGED;
                break;
            }
            const VT *pold = pb[it & 1];
            VT *pnew = pb[(it & 1) ^ 1];
            const VT bt = (VT)beta;
            // p = r + beta p over this CTA's rows, then a cluster barrier: the
            // SpMV gathers one vector (random column patterns make every
            // gathered element its own memory request)
            for (int i = ra + tid; i < rb; i += BNT) {
                if constexpr (MIX) pnew[i] = fmaf(bt, pold[i], r[i]);
                else pnew[i] = fma(bt, pold[i], r[i]);
            }
            cl.sync();
            const VT *pn_c = pnew;
            auto psrc = [=](int c) -> VT { return pn_c[c]; };
            double loc = 0.0;
            auto emit = [&](int i, VT pn, double y) {
                q[i] = (VT)y;
                loc += (double)pn * (double)(VT)y;
            };
            // the CTA's row chunks stream through two shared-memory stages
            // (bulk copies, completion on an mbarrier); every wait is bounded
            // and voted CTA-wide, and a failure is voted cluster-wide below
            bool fail = false;
            // thread 0 keeps the bounds of the next chunk to issue in registers,
            // loaded one issue ahead
            BChunk nxt;
            if (tid == 0) {
                for (int j = 0; j < BNS && cl0 + j < cl1; j++) b_issue<MIX>(a, S, rp_base, z0, b_chunk(a, sys, cl0 + j), j);
                if (cl0 + BNS < cl1) nxt = b_chunk(a, sys, cl0 + BNS);
            }
            __syncthreads();
            for (int c = cl0; c < cl1; c++) {
                const int k = (c - cl0) % BNS;
                const bool w = mbar_wait_bounded(&S.bar[k], use[k] & 1u, a.queue + 1, a.budget_ns);
                use[k]++;
                if (w) {
                    const BHdr &h = S.hdr[k];
                    const unsigned char *st = S.stage[k];
                    const int *rps = (const int *)(st + BOFF_RP + h.sh_rp);  // rowptr[h.r0 + j]
                    const int nr = h.r1 - h.r0;
                    // the trip count is the same for every lane (shuffles inside)
                    for (int qb = 0; qb < nr; qb += 2 * GPB) {
                        const int q0 = qb + grp, q1 = qb + GPB + grp;
                        // the rows' own p values are loaded before the row sums
                        VT pn0 = (VT)0, pn1 = (VT)0;
                        if (lane == 0) {
                            if (q0 < nr) pn0 = psrc(h.r0 + q0);
                            if (q1 < nr) pn1 = psrc(h.r0 + q1);
                        }
                        RowPair rr;
                        rr.a0 = q0 < nr ? rps[q0] : 0;
                        rr.e0 = q0 < nr ? rps[q0 + 1] : 0;
                        rr.a1 = q1 < nr ? rps[q1] : 0;
                        rr.e1 = q1 < nr ? rps[q1 + 1] : 0;
                        double y0, y1;
                        if (h.direct) {
                            row_dot2<L, MIX, decltype(psrc), true>(rr, col, val, val32, lane, psrc, y0, y1);
                        } else {
                            rr.a0 -= h.e0;
                            rr.e0 -= h.e0;
                            rr.a1 -= h.e0;
                            rr.e1 -= h.e0;
                            row_dot2<L, MIX, decltype(psrc), false>(
                                rr, (const int *)(st + BOFF_COL + h.sh_col), (const double *)(st + BOFF_VAL + h.sh_val),
                                (const float *)(st + BOFF_VAL + h.sh_val), lane, psrc, y0, y1);
                        }
                        if (lane == 0) {
                            if (q0 < nr) emit(h.r0 + q0, pn0, y0);
                            if (q1 < nr) emit(h.r0 + q1, pn1, y1);
                        }
                    }
                }
                if (!__syncthreads_and(w)) {
                    fail = true;
                    // this stage and the later ones may still be landing
                    mbar_drain(&S.bar[k], (use[k] - 1u) & 1u, a.queue + 1, a.budget_ns);
                    for (int j = 1; j < BNS && c + j < cl1; j++) {
                        const int kj = (c + j - cl0) % BNS;
                        mbar_drain(&S.bar[kj], use[kj] & 1u, a.queue + 1, a.budget_ns);
                        use[kj]++;
                    }
                    break;
                }
                if (tid == 0 && c + BNS < cl1) {
                    b_issue<MIX>(a, S, rp_base, z0, nxt, k);
                    if (c + BNS + 1 < cl1) nxt = b_chunk(a, sys, c + BNS + 1);
                }
            }
            if (tid == 0) s_fail = fail ? 1 : 0;
            const double pq = cluster_sum(cl, loc, &s_slot[2], s_warp);
            int any_fail = 0;
            for (unsigned kk = 0; kk < ncta; kk++) any_fail |= *cl.map_shared_rank(&s_fail, kk);
            if (any_fail) {
                status = MF_ERR_TIMEOUT;
                break;
            }
            if (!(pq != 0.0) || !isfinite(pq)) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
            const double alpha = rho / pq;
            loc = 0.0;
            for (int i = ra + tid; i < rb; i += BNT) {
                if (MIX) {
                    xlo[i] = fmaf((float)alpha, (float)pnew[i], (float)xlo[i]);
                    const float ri = fmaf(-(float)alpha, (float)q[i], (float)r[i]);
                    r[i] = ri;
                    loc += (double)ri * (double)ri;
                } else {
                    x[i] = fma(alpha, (double)pnew[i], x[i]);
                    const double ri = fma(-alpha, (double)q[i], (double)r[i]);
                    r[i] = ri;
                    loc += ri * ri;
                }
            }
            double rho_new = cluster_sum(cl, loc, &s_slot[3], s_warp);
            it++;
            if (MIX && (sqrt(rho_new) <= a.delta * rmax || sqrt(rho_new) <= a.tol * nb)) {
                for (int i = ra + tid; i < rb; i += BNT) {
                    x[i] += (double)xlo[i];
                    xlo[i] = (VT)0;
                }
                cl.sync();
                loc = 0.0;
                const double *xh = x;
                auto xsrc = [=](int c) -> double { return xh[c]; };
                for (int base = ra; base < rb; base += 2 * GPB) {
                    const int i0 = base + grp < rb ? base + grp : -1;
                    const int i1 = base + GPB + grp < rb ? base + GPB + grp : -1;
                    double y0, y1;
                    row_dot2<L, false>(row_pair(rp, i0, i1), col, val, val32, lane, xsrc, y0, y1);
                    if (lane == 0) {
                        if (i0 >= 0) {
                            const VT rv = (VT)(b[i0] - y0);
                            r[i0] = rv;
                            loc += (double)rv * (double)rv;
                        }
                        if (i1 >= 0) {
                            const VT rv = (VT)(b[i1] - y1);
                            r[i1] = rv;
                            loc += (double)rv * (double)rv;
                        }
                    }
                }
                rho_new = cluster_sum(cl, loc, &s_slot[1], s_warp);
                rmax = sqrt(rho_new);
                refs++;
            }
            beta = rho_new / rho;
            rho = rho_new;
            relres = sqrt(rho) / nb;
        }
        if (MIX && status != MF_OK) {
            for (int i = ra + tid; i < rb; i += BNT) x[i] += (double)xlo[i];
        }
        if (rank == 0 && tid == 0) {
            a.iters[sys] = it;
            a.refs[sys] = refs;
            a.status[sys] = status;
            a.relres[sys] = relres;
        }
        cl.sync();  // the cluster's last writes land before the next system
    }
}

template <int L, bool MIX>
int batched_ctas(int count, int cluster)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // clusters of 16 CTAs are above the portable size: allowed explicitly
    if (cluster > 8) cudaFuncSetAttribute(k_batched_cg<L, MIX>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_batched_cg<L, MIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batched_cg<L, MIX>, BNT, sizeof(BSmem));
    int ctas = sms * (per > 0 ? per : 1);
    ctas = (ctas / cluster) * cluster;
    const int want = count * cluster;
    if (ctas > want) ctas = want;
    if (ctas < cluster) ctas = cluster;
    return ctas;
}

template <bool MIX>
int batched_ctas_l(int lanes, int count, int cluster)
{
    switch (lanes) {
    case 4: return batched_ctas<4, MIX>(count, cluster);
    case 8: return batched_ctas<8, MIX>(count, cluster);
    case 16: return batched_ctas<16, MIX>(count, cluster);
    default: return batched_ctas<32, MIX>(count, cluster);
    }
}

// ctas: computed before any stream capture (batched_ctas)
template <int L, bool MIX>
mf_status launch_batched(const BatchArgs &a, int cluster, int ctas, cudaStream_t s)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(BNT);
    cfg.dynamicSmemBytes = sizeof(BSmem);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // enough clusters to fill the GPU (the work queue balances them)
    cfg.gridDim = dim3(ctas);
    note_launch();
    MF_CUDA(cudaLaunchKernelEx(&cfg, k_batched_cg<L, MIX>, a));
    return MF_OK;
}

template <bool MIX>
mf_status launch_batched_l(int lanes, const BatchArgs &a, int cluster, int ctas, cudaStream_t s)
{
    switch (lanes) {
    case 4: return launch_batched<4, MIX>(a, cluster, ctas, s);
    case 8: return launch_batched<8, MIX>(a, cluster, ctas, s);
    case 16: return launch_batched<16, MIX>(a, cluster, ctas, s);
    default: return launch_batched<32, MIX>(a, cluster, ctas, s);
    }
}

__global__ void k_batch_resid(int count, const int *n, const long long *row0, const long long *nz0,
                              const int *rowptr, const int *col, const double *val, const double *b, const double *x,
                              double *out)
{
    // one CTA per system: ||b - A x|| / ||b|| in FP64
    __shared__ double s_warp[8];
    for (int sys = blockIdx.x; sys < count; sys += gridDim.x) {
        const int nn = n[sys];
        const long long r0 = row0[sys], z0 = nz0[sys];
        const int *rp = rowptr + r0 + sys;
        double rr = 0.0, bb = 0.0;
        for (int i = threadIdx.x; i < nn; i += blockDim.x) {
            double y = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; k++) y += val[z0 + k] * x[r0 + col[z0 + k]];
            const double d = b[r0 + i] - y;
            rr += d * d;
            bb += b[r0 + i] * b[r0 + i];
        }
        rr = block_sum<256>(rr, s_warp);
        bb = block_sum<256>(bb, s_warp);
        if (threadIdx.x == 0) out[sys] = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
        __syncthreads();
    }
}

__global__ void k_to_f32(long long n, const double *in, float *out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" {

mf_status mf_batch_create(int count, const int *n, const int *const *rowptr, const int *const *colidx,
                          const double *const *val, mf_batch *out)
{
    if (!out || count <= 0 || !n || !rowptr || !colidx || !val) return MF_ERR_INVALID_ARG;
    *out = nullptr;
    mf_batch bt = new mf_batch_s();
    bt->count = count;
    bt->n.assign(n, n + count);
    std::vector<long long> row0(count), nz0(count);
    long long rows = 0, nz = 0;
    for (int s = 0; s < count; s++) {
        if (n[s] <= 0 || !rowptr[s] || rowptr[s][0] != 0) {
            delete bt;
            set_last_error("mf_batch_create: system %d has no rows or rowptr[0] != 0", s);
            return MF_ERR_INVALID_ARG;
        }
        row0[s] = rows;
        nz0[s] = nz;
        rows += n[s];
        nz += rowptr[s][n[s]];
    }
    bt->rows_total = rows;
    bt->nnz_total = nz;
    bt->row0 = row0;
    // host staging of the concatenated CSR (validated)
    std::vector<int> hrp((size_t)rows + count), hcol((size_t)nz);
    std::vector<double> hval((size_t)nz);
    for (int s = 0; s < count; s++) {
        memcpy(&hrp[row0[s] + s], rowptr[s], sizeof(int) * (n[s] + 1));
        const int e = rowptr[s][n[s]];
        for (int k = 0; k < e; k++) {
            const int c = colidx[s][k];
            if (c < 0 || c >= n[s]) {
                delete bt;
                set_last_error("mf_batch_create: system %d column %d outside [0, %d)", s, c, n[s]);
                return MF_ERR_INVALID_ARG;
            }
        }
        memcpy(&hcol[nz0[s]], colidx[s], sizeof(int) * e);
        memcpy(&hval[nz0[s]], val[s], sizeof(double) * e);
    }
    // row chunks of each system: at most BCR rows and BCE entries (a longer
    // row alone); per system nch + 1 row starts and entry offsets
    std::vector<int> sc(count + 1), crow, cent;
    for (int s = 0; s < count; s++) {
        sc[s] = (int)(crow.size() - s);
        const int *rp = rowptr[s];
        int r = 0;
        while (r < n[s]) {
            crow.push_back(r);
            cent.push_back(rp[r]);
            const int r_start = r;
            r++;
            while (r < n[s] && r - r_start < BCR && rp[r + 1] - rp[r_start] <= BCE) r++;
        }
        crow.push_back(n[s]);
        cent.push_back(rp[n[s]]);
    }
    sc[count] = (int)(crow.size() - count);
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    auto fail = [&](cudaError_t e) {
        set_last_error("mf_batch_create: %s", cudaGetErrorString(e));
        mf_batch_destroy(bt);
        return e == cudaErrorMemoryAllocation ? MF_ERR_NO_MEMORY : MF_ERR_CUDA;
    };
    cudaError_t e = cudaSuccess;
#define BT_ALLOC(p, bytes) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    BT_ALLOC(bt->d_order, sizeof(int) * count);
    BT_ALLOC(bt->d_n, sizeof(int) * count);
    BT_ALLOC(bt->d_row0, sizeof(long long) * count);
    BT_ALLOC(bt->d_nz0, sizeof(long long) * count);
    BT_ALLOC(bt->d_rowptr, sizeof(int) * (rows + count + 8));  // slack: 16-byte bulk-copy rounding
    BT_ALLOC(bt->d_sc, sizeof(int) * (count + 1));
    BT_ALLOC(bt->d_crow, sizeof(int) * crow.size());
    BT_ALLOC(bt->d_cent, sizeof(int) * cent.size());
    BT_ALLOC(bt->d_col, sizeof(int) * (nz + 4));
    BT_ALLOC(bt->d_val, sizeof(double) * (nz + 2));
    BT_ALLOC(bt->d_val32, sizeof(float) * (nz + 4));
    BT_ALLOC(bt->d_iters, sizeof(int) * count);
    BT_ALLOC(bt->d_refs, sizeof(int) * count);
    BT_ALLOC(bt->d_status, sizeof(int) * count);
    BT_ALLOC(bt->d_relres, sizeof(double) * count * 2);
    BT_ALLOC(bt->d_queue, sizeof(int) * 4);
#undef BT_ALLOC
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_order, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_n, n, sizeof(int) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_row0, row0.data(), sizeof(long long) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_nz0, nz0.data(), sizeof(long long) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_rowptr, hrp.data(), sizeof(int) * (rows + count), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_sc, sc.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_crow, crow.data(), sizeof(int) * crow.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bt->d_cent, cent.data(), sizeof(int) * cent.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nz) e = cudaMemcpy(bt->d_col, hcol.data(), sizeof(int) * nz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nz) e = cudaMemcpy(bt->d_val, hval.data(), sizeof(double) * nz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nz) {
        k_to_f32<<<1184, 256>>>(nz, bt->d_val, bt->d_val32);
        note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(e);
    *out = bt;
    return MF_OK;
}

mf_status mf_batch_destroy(mf_batch bt)
{
    if (!bt) return MF_OK;
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    void *bufs[] = {bt->d_order, bt->d_n, bt->d_row0, bt->d_nz0, bt->d_rowptr, bt->d_col, bt->d_val, bt->d_val32,
                    bt->d_iters, bt->d_refs, bt->d_status, bt->d_relres, bt->work, bt->d_queue, bt->d_sc,
                    bt->d_crow, bt->d_cent};
    for (void *p : bufs)
        if (p) cudaFree(p);
    delete bt;
    return MF_OK;
}

mf_status mf_batch_info(mf_batch bt, long long *rows_total, long long *nnz_total, const long long **row_offsets)
{
    if (!bt) return MF_ERR_INVALID_ARG;
    if (rows_total) *rows_total = bt->rows_total;
    if (nnz_total) *nnz_total = bt->nnz_total;
    if (row_offsets) *row_offsets = bt->row0.data();
    return MF_OK;
}

static mf_status batch_work(mf_batch bt, bool mixed)
{
    const size_t rows = (size_t)bt->rows_total + 16;
    const size_t need = rows * 8 * 5 + 1024;
    (void)mixed;
    if (bt->work_bytes >= need) return MF_OK;
    if (bt->work) cudaFree(bt->work);
    bt->work = nullptr;
    bt->work_bytes = 0;
    MF_CUDA(cudaMalloc(&bt->work, need));
    bt->work_bytes = need;
    return MF_OK;
}

// Enqueues one batched solve.  Nothing here allocates or queries the device:
// batch_work() and batched_ctas_l() run before (outside any stream capture).
static mf_status batch_enqueue(mf_batch bt, const double *b, double *x, const mf_solve_opts &o, int lanes,
                               int cluster, int ctas, cudaStream_t s)
{
    const bool mixed = o.policy != MF_POLICY_FP64;
    const size_t rows = (size_t)bt->rows_total + 16;
    char *w = (char *)bt->work;
    BatchArgs a;
    a.count = bt->count;
    a.order = bt->d_order;
    a.n = bt->d_n;
    a.row0 = bt->d_row0;
    a.nz0 = bt->d_nz0;
    a.rowptr = bt->d_rowptr;
    a.col = bt->d_col;
    a.val = bt->d_val;
    a.val32 = bt->d_val32;
    a.b = b;
    a.x = x;
    a.r = w;
    a.p0 = w + rows * 8;
    a.p1 = w + rows * 16;
    a.q = w + rows * 24;
    a.xlo = w + rows * 32;
    a.queue = bt->d_queue;
    a.iters = bt->d_iters;
    a.refs = bt->d_refs;
    a.status = bt->d_status;
    a.relres = bt->d_relres;
    a.maxiter = o.maxiter;
    a.tol = o.tol;
    a.delta = (o.refine_delta > 0 && o.refine_delta < 1) ? o.refine_delta : 0.1;
    a.budget_ns = (unsigned long long)(o.wait_budget_s * 1e9);
    a.sc = bt->d_sc;
    a.crow = bt->d_crow;
    a.cent = bt->d_cent;
    MF_CUDA(cudaMemsetAsync(bt->d_queue, 0, sizeof(int) * 2, s));  // queue head, stage-wait status
    if (mixed) MF_TRY(launch_batched_l<true>(lanes, a, cluster, ctas, s));
    else MF_TRY(launch_batched_l<false>(lanes, a, cluster, ctas, s));
    k_batch_resid<<<std::min(bt->count, 1184), 256, 0, s>>>(bt->count, bt->d_n, bt->d_row0, bt->d_nz0, bt->d_rowptr,
                                                           bt->d_col, bt->d_val, b, x, bt->d_relres + bt->count);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

mf_status mf_batch_tune(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int *lanes_out,
                        int *cluster_out, void *stream);

mf_status mf_batch_cg_solve(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int use_graph,
                            mf_batch_report *report, void *stream)
{
    if (!bt || !b || !x) return MF_ERR_INVALID_ARG;
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    if (opts) o = *opts;
    if (o.tol <= 0 || o.maxiter <= 0) {
        set_last_error("batched CG needs tol > 0 and maxiter > 0");
        return MF_ERR_INVALID_ARG;
    }
    if (o.precond) {
        set_last_error("batched CG: no preconditioner");
        return MF_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int lanes = bt->tuned_lanes ? bt->tuned_lanes : 8;
    int cluster = bt->tuned_cluster ? bt->tuned_cluster : 4;
    if (const char *e = getenv("MF_BATCH_LANES")) lanes = atoi(e);
    if (const char *e = getenv("MF_BATCH_CLUSTER")) cluster = atoi(e);
    if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) lanes = 8;
    if (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16) cluster = 4;
    const bool mixed = o.policy != MF_POLICY_FP64;
    MF_TRY(batch_work(bt, mixed));
    const int ctas = mixed ? batched_ctas_l<true>(lanes, bt->count, cluster) : batched_ctas_l<false>(lanes, bt->count, cluster);
    cudaEvent_t e0, e1;
    MF_CUDA(cudaEventCreate(&e0));
    MF_CUDA(cudaEventCreate(&e1));
    MF_CUDA(cudaEventRecord(e0, s));
    const int key[6] = {lanes, cluster, o.policy, (int)(o.tol * 1e15), o.maxiter, 1};
    if (use_graph) {
        // one graph per (buffers, configuration): replayed on later calls
        if (!bt->graph || bt->graph_b != b || bt->graph_x != x || memcmp(key, bt->graph_key, sizeof(key))) {
            if (bt->graph) cudaGraphExecDestroy(bt->graph);
            bt->graph = nullptr;
            cudaStream_t cs;
            MF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaGraph_t g;
            MF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            mf_status st = batch_enqueue(bt, b, x, o, lanes, cluster, ctas, cs);
            cudaError_t ce = cudaStreamEndCapture(cs, &g);
            cudaStreamDestroy(cs);
            if (st != MF_OK || ce != cudaSuccess) {
                if (ce == cudaSuccess) cudaGraphDestroy(g);
                cudaGetLastError();
                if (st != MF_OK) return st;
                MF_CUDA(ce);
            }
            MF_CUDA(cudaGraphInstantiate(&bt->graph, g, 0));
            cudaGraphDestroy(g);
            bt->graph_b = b;
            bt->graph_x = x;
            memcpy(bt->graph_key, key, sizeof(key));
        }
        MF_CUDA(cudaGraphLaunch(bt->graph, s));
        note_launch(2);  // the graph's kernels: the batched CG and the residual check
    } else {
        MF_TRY(batch_enqueue(bt, b, x, o, lanes, cluster, ctas, s));
    }
    MF_CUDA(cudaEventRecord(e1, s));
    MF_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int count = bt->count;
    std::vector<int> it(count), rf(count), stt(count);
    std::vector<double> rr(count * 2);
    MF_CUDA(cudaMemcpy(it.data(), bt->d_iters, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(rf.data(), bt->d_refs, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(stt.data(), bt->d_status, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(rr.data(), bt->d_relres, sizeof(double) * count * 2, cudaMemcpyDeviceToHost));
    mf_status worst = MF_OK;
    long long iters = 0;
    double maxrr = 0;
    int maxit = 0, refs = 0, failed = 0;
    for (int k = 0; k < count; k++) {
        iters += it[k];
        maxit = std::max(maxit, it[k]);
        refs += rf[k];
        maxrr = std::max(maxrr, rr[count + k]);
        if (stt[k] != MF_OK) {
            failed++;
            if (worst == MF_OK) worst = (mf_status)stt[k];
        }
    }
    if (report) {
        report->systems = count;
        report->failed = failed;
        report->iterations_total = iters;
        report->iterations_max = maxit;
        report->refinements_total = refs;
        report->relres_true_max = maxrr;
        report->kernel_ms = ms;
        report->lanes_per_row = lanes;
        report->cluster_ctas = cluster;
        report->status = worst;
    }
    if (worst != MF_OK) set_last_error("%d of %d systems did not converge", failed, count);
    return worst;
}

mf_status mf_batch_results(mf_batch bt, int *iterations, double *relres_true)
{
    if (!bt) return MF_ERR_INVALID_ARG;
    if (iterations) MF_CUDA(cudaMemcpy(iterations, bt->d_iters, sizeof(int) * bt->count, cudaMemcpyDeviceToHost));
    if (relres_true)
        MF_CUDA(cudaMemcpy(relres_true, bt->d_relres + bt->count, sizeof(double) * bt->count, cudaMemcpyDeviceToHost));
    return MF_OK;
}

// Autotuner: times every (lanes per row, cluster size) pair on this batch
// and keeps the fastest; the choice is returned and kept on the handle.
mf_status mf_batch_tune(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int *lanes_out,
                        int *cluster_out, void *stream)
{
    if (!bt || !b || !x) return MF_ERR_INVALID_ARG;
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    if (opts) o = *opts;
    const int lanes_c[] = {4, 8, 16, 32};
    const int clus_c[] = {1, 2, 4, 8, 16};
    float best = 1e30f;
    int bl = 8, bc = 4;
    cudaStream_t s = (cudaStream_t)stream;
    const bool mixed = o.policy != MF_POLICY_FP64;
    MF_TRY(batch_work(bt, mixed));
    for (int li : lanes_c)
        for (int ci : clus_c) {
            const int ctas = mixed ? batched_ctas_l<true>(li, bt->count, ci) : batched_ctas_l<false>(li, bt->count, ci);
            cudaEvent_t e0, e1;
            MF_CUDA(cudaEventCreate(&e0));
            MF_CUDA(cudaEventCreate(&e1));
            MF_CUDA(cudaEventRecord(e0, s));
            mf_status st = batch_enqueue(bt, b, x, o, li, ci, ctas, s);
            MF_CUDA(cudaEventRecord(e1, s));
            MF_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            if (st == MF_OK && ms < best) {
                best = ms;
                bl = li;
                bc = ci;
            }
        }
    bt->tuned_lanes = bl;
    bt->tuned_cluster = bc;
    if (lanes_out) *lanes_out = bl;
    if (cluster_out) *cluster_out = bc;
    return MF_OK;
}

mf_status mf_batch_set_schedule(mf_batch bt, int lanes, int cluster)
{
    if (!bt || (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) ||
        (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16))
        return MF_ERR_INVALID_ARG;
    bt->tuned_lanes = lanes;
    bt->tuned_cluster = cluster;
    return MF_OK;
}

}  // extern "C"
