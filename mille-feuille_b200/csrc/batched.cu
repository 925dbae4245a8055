// batched.cu -- many independent CG solves of uneven size in one launch,
// with per-chunk precision classes chosen on the chip.
//
// No reference counterpart: the reference solves one system per launch.
// Design for B200: the systems are sorted by size and handed out by a device
// work queue to thread-block clusters; a cluster of C CTAs (one per SM)
// solves one system at a time.  A system's rows are cut into chunks and the
// chunks are split across the cluster's CTAs; every dot product is reduced
// through distributed shared memory with a hardware cluster barrier -- no
// grid-wide synchronisation, so small systems cost no more than their own
// iterations.
//
// Random column patterns make the SpMV gather-bound when the gathered vector
// comes from L1/L2: every lane's element is its own cache line, about one
// line per cycle per SM.  The matrix is therefore stored in column panels of
// PW = 32768 columns (16-bit column offsets within the panel, rows of each
// panel in CSR), and the mixed-precision kernel copies the panel's slice of p
// (FP32, 128 KB) into shared memory before it streams the panel's chunks:
// the gathers hit shared memory (about 8 lanes per cycle for random
// addresses).  A chunk is a range of rows with at most BCE entries in every
// panel; for each (chunk, panel) pair its row pointers, columns and values
// arrive by bulk copies in one of NS = 3 shared-memory stages, produced by
// warp 0 and consumed, in the mixed kernel, by a group of five warps per
// stage (the FP64 kernel's fifteen consumer warps all take every pass).  A
// mixed pass sums its rows in two phases: the products of consecutive
// entries on consecutive lanes, written over the staged values, then one
// lane per row adding its products in entry order.  The row sums of the
// panels are added in panel order (partial sums kept in q).  The FP64 kernel
// (the FP64 policy and trace collection) gathers p from global memory.
//
// Values are held three times: FP64 (reliable updates, FP64 policy), FP32,
// and FP16 scaled per row by a power of two (the row's largest
// off-diagonal magnitude maps into [2^14, 2^15)) with the diagonal taken out
// and kept in FP32 beside the row scale.  A mixed-precision solve reads each
// chunk in its working class -- FP32 (4 + 2 bytes per entry) or FP16 (one
// 4-byte word per entry: the value bits and the column offset) -- and
// accumulates in FP32; FP64 dot products, FP64 reliable updates
// r = b - A x from the FP64 values, convergence judged on that FP64
// residual.
//
// Classes per chunk, decided inside the persistent kernel by the CTA that
// owns the chunk (no host round trip):
//   STATIC   the value-range class: FP16 when every value of the chunk is
//            exactly representable (scaled FP16 off-diagonals, FP32
//            diagonal), else FP32; fixed for the solve.
//   RULE     after every p update, the reference's partial-convergence
//            thresholds (src/main-cg-mixed.cu:415-460) on the chunk's own
//            rows: v = max |p_new - p_old| in FP64; v > 1e-6 (FP64 and FP32
//            decisions) -> FP32, else FP16 (the FP16, INT8 and BYPASS
//            decisions: rows cannot be skipped in a row-chunk layout, and
//            the values are not integers).
//   LEARNED  at the first iteration and at every reliable update, the MLP
//            (16 chunk features -> 32 -> 32 -> 4, BF16 weights, FP32
//            accumulation) of an attached mf_learned: FP16 where it is at
//            least 90 % sure the chunk's label is FP16 or narrower.
// RULE and LEARNED fall back to the static classes for the rest of a
// system's solve when a reliable update finds the FP64 residual above half
// of the previous one (the recurrence claimed a tenfold drop).
// A chunk whose rows' FP16 scales fall outside FP32's range stays FP32.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include <type_traits>

#include "mf_internal.h"
#include "policy_net.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

namespace mf {
namespace {
constexpr int PW = 32768;   // columns per storage panel (16-bit offsets)
#ifndef MF_BATCH_BCE
#define MF_BATCH_BCE 4096
#endif
#ifndef MF_BATCH_BCR
#define MF_BATCH_BCR 256
#endif
constexpr int BCE = MF_BATCH_BCE;   // entries of a (chunk, panel) stage
constexpr int BCR = MF_BATCH_BCR;   // rows of a chunk
}  // namespace
}  // namespace mf

struct mf_batch_s {
    int count = 0;
    long long rows_total = 0, nnz_total = 0;
    int nchunks = 0, npanels = 0;
    std::vector<int> n;           // rows per system (caller order)
    std::vector<long long> row0;  // first row of each system (caller order)
    std::vector<long long> nz0;   // first entry of each system
    int *d_order = nullptr;       // systems by descending size
    long long *d_row0 = nullptr;
    int *d_n = nullptr, *d_pan0 = nullptr, *d_npan = nullptr;  // per system: first panel, panels
    long long *d_prow0 = nullptr; // per panel: first of its n+1 row pointers
    long long *d_pent0 = nullptr; // per panel (+1): first entry
    int *d_prow = nullptr;        // panel row pointers, relative to the panel's first entry
    uint16_t *d_col = nullptr;    // column offset within the panel
    double *d_val = nullptr;
    float *d_val32 = nullptr;
    __half *d_val16 = nullptr;    // row-scaled, diagonal entries 0
    uint32_t *d_cv16 = nullptr;   // FP16 value bits << 16 | column offset (one word per entry)
    float *d_rscale = nullptr;    // per row: scale of the FP16 values
    float *d_diag32 = nullptr;    // per row: diagonal (sum of the row's diagonal entries)
    // row chunks of every system
    int *d_sc = nullptr;          // [count+1] first chunk of each system
    int *d_crow = nullptr;        // per system nch+1 chunk row starts (relative rows), at sc[s] + s
    int *d_cent = nullptr;        // the same chunks' entries over all panels (sc[s] + s, scanned)
    unsigned char *d_ccls = nullptr;         // [chunks] working class (0 FP32, 1 FP16)
    unsigned char *d_ccls_static = nullptr;  // [chunks] bit 0: FP16 exact, bit 1: FP16 allowed
    float *d_cstat = nullptr;     // [chunks][NCSTAT] static features
    float *d_cdyn = nullptr;      // [chunks][NCDYN] checkpoint statistics
    // per-system results
    int *d_iters = nullptr, *d_refs = nullptr, *d_status = nullptr;
    double *d_relres = nullptr;
    unsigned long long *d_sysstat = nullptr;  // [count][3] matrix bytes streamed, FP16 chunk passes, chunk passes
    void *work = nullptr;
    size_t work_bytes = 0;
    int *d_queue = nullptr;
    // CUDA graph of the last solve configuration
    cudaGraphExec_t graph = nullptr;
    const void *graph_b = nullptr;
    void *graph_x = nullptr;
    int graph_key[7] = {0, 0, 0, 0, 0, 0, 0};
    int tuned_lanes = 0, tuned_cluster = 0;
    int static_fp16_chunks = 0, fp16_allowed_chunks = 0;
    struct mf_policy_s *policy = nullptr;     // LEARNED solves
};

namespace mf {

mf_status policy_sample_buffers(struct mf_policy_s *p, long long max_samples, float **x, unsigned char **y,
                                long long *n);
mf_status policy_sample_commit(struct mf_policy_s *p, long long n_total);
const __nv_bfloat16 *policy_weights(struct mf_policy_s *p);

namespace {

constexpr int BNT = 512;
constexpr int BNW = BNT / 32;
constexpr int NCSTAT = 6;   // static chunk features 0-4, and max |a| of the chunk
constexpr int NCDYN = 10;   // [0..3] raw maxima |r|, |p|, |dp|, |q|; [4..7] previous features 6..9; [8] label ratio
constexpr float LEARN_CONF = 0.9f;   // FP16 when P(label <= FP16) >= this
constexpr double LABEL_TAU = 0.015625;  // label FP16: ||dq_c|| <= 2^-6 ||q_c|| (FP16 perturbation of A p)

struct BatchArgs {
    int count;
    const int *order;
    const int *n, *pan0, *npan;
    const long long *row0, *prow0, *pent0;
    const int *prow;
    const uint16_t *col;
    const double *val;
    const float *val32;
    const __half *val16;
    const uint32_t *cv16;
    const float *rscale, *diag32;
    const double *b;
    double *x;
    void *r, *p0, *p1, *q, *xlo;  // workspace vectors (rows_total each)
    const int *sc, *crow, *cent;   // row chunks
    unsigned char *ccls;
    const unsigned char *ccls_static;
    const float *cstat;
    float *cdyn;
    int *queue;
    int *iters, *refs, *status;
    double *relres;
    unsigned long long *sysstat;
    int maxiter;
    double tol;
    double delta;
    unsigned long long budget_ns;  // bound of every shared-memory stage wait
    unsigned backoff_ns;           // sleep between retries of a stage wait
    int rowsum;                    // mixed passes: 0 two-phase row sums, 1 lane groups per row
    int policy;
    const __nv_bfloat16 *mlp_w;    // LEARNED: the network's BF16 weights
    // trace collection (FP64 solves): samples every collect_every iterations
    int collect_every, collect_stride;
    unsigned collect_salt;
    float *cx;
    unsigned char *cy;
    unsigned long long *ccount;
    long long ccap;
};

// One system's view of the panel storage.
struct SysView {
    int n, npan, gp0;
    long long r0;
};

__device__ __forceinline__ SysView sys_view(const BatchArgs &a, int sys)
{
    SysView v;
    v.n = a.n[sys];
    v.npan = a.npan[sys];
    v.gp0 = a.pan0[sys];
    v.r0 = a.row0[sys];
    return v;
}

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

// Cluster-wide maximum of two non-negative values (exact, so any order).
__device__ __forceinline__ void cluster_max2(cg::cluster_group &cl, float &a, float &b, float *slot2, float *s_warp2)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        s_warp2[2 * (threadIdx.x >> 5)] = a;
        s_warp2[2 * (threadIdx.x >> 5) + 1] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float ma = 0.f, mb = 0.f;
        for (int w = 0; w < BNW; w++) {
            ma = fmaxf(ma, s_warp2[2 * w]);
            mb = fmaxf(mb, s_warp2[2 * w + 1]);
        }
        slot2[0] = ma;
        slot2[1] = mb;
    }
    cl.sync();
    a = 0.f;
    b = 0.f;
    for (unsigned k = 0; k < cl.num_blocks(); k++) {
        const float *o = cl.map_shared_rank(slot2, k);
        a = fmaxf(a, o[0]);
        b = fmaxf(b, o[1]);
    }
}

struct BHdr {
    int r0, r1, e0, direct;   // rows [r0, r1), first entry e0 (relative to the panel)
    int sh_rp, sh_col, sh_val, cls;
    int panel, sh_rs, sh_dg, pad0;
    long long ebase;          // the panel's first entry (global)
};

// Stages in flight per CTA.  The mixed kernels stage at most 4 + 2 bytes
// per entry (FP32 values, 16-bit columns); their consumer warps form
// MF_BATCH_GROUPS groups, group g consuming the stages k with k % groups = g.
#ifndef MF_BATCH_STAGES_MIX
#define MF_BATCH_STAGES_MIX 3
#endif
#ifndef MF_BATCH_GROUPS
#define MF_BATCH_GROUPS 3
#endif
#ifndef MF_BATCH_STAGES_FP64
#define MF_BATCH_STAGES_FP64 3
#endif

// Shared-memory stage of one (chunk, panel) pair: row pointers, columns,
// values.
template <bool MIX>
struct Stage {
    static constexpr int NS = MIX ? MF_BATCH_STAGES_MIX : MF_BATCH_STAGES_FP64;
    static constexpr int VB = MIX ? 4 : 8;  // widest stored value
    static constexpr int OFF_RP = 0;
    static constexpr int OFF_COL = ((BCR + 1) * 4 + 32 + 15) & ~15;
    static constexpr int OFF_VAL = OFF_COL + ((BCE * 2 + 32 + 15) & ~15);
    static constexpr int OFF_RS = OFF_VAL + ((BCE * VB + 32 + 15) & ~15);  // FP16 passes: row scales
    static constexpr int OFF_DG = OFF_RS + ((BCR * 4 + 32 + 15) & ~15);    // FP16 passes: FP32 diagonals
    static constexpr int SIZE = OFF_DG + ((BCR * 4 + 32 + 15) & ~15);
    static_assert(OFF_COL % 16 == 0 && OFF_VAL % 16 == 0 && SIZE % 16 == 0, "stage regions 16-byte aligned");
    static_assert((BCR + 1) * 4 + 32 <= OFF_COL, "row pointers fit");
    static_assert(NS >= 1 && NS <= 8, "stage phases kept in a byte");
};

template <bool MIX>
struct BSmem {
    unsigned char stage[Stage<MIX>::NS][Stage<MIX>::SIZE];
    BHdr hdr[Stage<MIX>::NS];
    uint64_t bar[Stage<MIX>::NS];    // stage full (the producer's copies landed)
    uint64_t empty[Stage<MIX>::NS];  // stage released by every consumer warp
    uint64_t pbar;                   // the p window's copy landed
    uint64_t wempty;                 // the p window released by every consumer warp
};

// dynamic shared memory: the stages, the p window (mixed kernel: a panel
// of p in FP32), the MLP weights as float and the per-warp feature rows
template <bool MIX>
struct SmemLayout {
    static constexpr size_t PWIN = (sizeof(BSmem<MIX>) + 15) & ~(size_t)15;
    static constexpr size_t PWIN_BYTES = MIX ? (size_t)PW * 4 + 32 : 0;
    static constexpr size_t W = PWIN + PWIN_BYTES;
    static constexpr size_t FEAT = W + sizeof(float) * ((PN_NPARAM + 3) & ~3);
    static constexpr size_t TOTAL = FEAT + sizeof(float) * BNW * PN_NF;
    static_assert(TOTAL <= 227 * 1024, "one CTA per SM");
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

// A (chunk, panel) pair: rows [r0, r1) of the system, entries [e0, e1) of
// the panel (relative to its first entry ebase), the chunk's class.
struct BChunk {
    int r0, r1, e0, e1, cls, panel;
    long long ebase, rpbase, rowbase;
};

__device__ __forceinline__ BChunk b_chunk(const BatchArgs &a, int sys, const SysView &v, int c, int k, bool mix)
{
    BChunk ch;
    ch.r0 = a.crow[c + sys];
    ch.r1 = a.crow[c + 1 + sys];
    ch.panel = k;
    ch.rpbase = a.prow0[v.gp0 + k];
    ch.ebase = a.pent0[v.gp0 + k];
    ch.e0 = a.prow[ch.rpbase + ch.r0];
    ch.e1 = a.prow[ch.rpbase + ch.r1];
    ch.cls = mix ? (int)a.ccls[c] : 0;
    ch.rowbase = v.r0;
    return ch;
}

// Algorithmic bytes of one (chunk, panel) pass in class `cls`.
template <bool MIX>
__device__ __forceinline__ unsigned long long chunk_bytes(const BChunk &ch)
{
    const unsigned long long ne = (unsigned long long)(ch.e1 - ch.e0), nr = (unsigned long long)(ch.r1 - ch.r0);
    const unsigned vb = MIX ? (ch.cls ? 2u : 4u) : 8u;
    return ne * (vb + 2) + (nr + 1) * 4 + (ch.cls ? nr * 8 : 0);
}

// Thread 0: stage pair `ch` into stage k.
template <bool MIX>
__device__ void b_issue(const BatchArgs &a, BSmem<MIX> &S, const BChunk &ch, int k)
{
    using SG = Stage<MIX>;
    BHdr &h = S.hdr[k];
    const int r0 = ch.r0, r1 = ch.r1, e0 = ch.e0, e1 = ch.e1;
    h.r0 = r0;
    h.r1 = r1;
    h.e0 = e0;
    h.direct = (e1 - e0 > BCE) ? 1 : 0;
    h.cls = ch.cls;
    h.panel = ch.panel;
    h.ebase = ch.ebase;
    const long long z0 = ch.ebase, rw = ch.rowbase;
    const bool h16 = MIX && ch.cls == 1;  // FP16 rows: packed (value, column) words, row scales and diagonals
    const int vb = MIX ? 4 : 8;  // FP16 passes: one 4-byte word per entry
    unsigned total = b_range_bytes(4 * (ch.rpbase + r0), 4 * (ch.rpbase + r1 + 1));
    if (!h.direct) {
        total += b_range_bytes(vb * (z0 + e0), vb * (z0 + e1));
        if (!h16) total += b_range_bytes(2 * (z0 + e0), 2 * (z0 + e1));
    }
    if (h16) total += 2 * b_range_bytes(4 * (rw + r0), 4 * (rw + r1));
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.bar[k], total);
    unsigned char *st = S.stage[k];
    b_add_range(st + SG::OFF_RP, (const unsigned char *)a.prow, 4 * (ch.rpbase + r0), 4 * (ch.rpbase + r1 + 1),
                &S.bar[k], h.sh_rp);
    if (h16) {
        b_add_range(st + SG::OFF_RS, (const unsigned char *)a.rscale, 4 * (rw + r0), 4 * (rw + r1), &S.bar[k], h.sh_rs);
        b_add_range(st + SG::OFF_DG, (const unsigned char *)a.diag32, 4 * (rw + r0), 4 * (rw + r1), &S.bar[k], h.sh_dg);
    }
    if (h.direct) return;
    if (!h16)
        b_add_range(st + SG::OFF_COL, (const unsigned char *)a.col, 2 * (z0 + e0), 2 * (z0 + e1), &S.bar[k], h.sh_col);
    const unsigned char *vsrc = MIX ? (h16 ? (const unsigned char *)a.cv16 : (const unsigned char *)a.val32)
                                    : (const unsigned char *)a.val;
    b_add_range(st + SG::OFF_VAL, vsrc, vb * (z0 + e0), vb * (z0 + e1), &S.bar[k], h.sh_val);
}

// L lanes per row: lanes stride over the row's entries (BU entries per lane
// loaded before any is used); the partials are combined with a fixed xor
// tree, so every run gives the same bits.  Two rows per lane group are in
// flight at once (a row with no entries: bounds 0, 0).
#ifndef MF_BATCH_BU
#define MF_BATCH_BU 4
#endif
constexpr int BU = MF_BATCH_BU;

// product loads in flight per lane in the two-phase row sums
#ifndef MF_BATCH_P1U
#define MF_BATCH_P1U 8
#endif
#define MF_PRAGMA(x) _Pragma(#x)
#define MF_UNROLL(n) MF_PRAGMA(unroll n)

struct RowPair {
    int a0, e0, a1, e1;
};

__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }

template <typename V>
__device__ __forceinline__ V ld_stream(const V *p)
{
    return __ldcs(p);
}
template <>
__device__ __forceinline__ __half ld_stream<__half>(const __half *p)
{
    return __ushort_as_half(__ldcs((const unsigned short *)p));
}

// Row sums of two rows; V is the stored value type (double, float, or the
// row-scaled __half).  FP64 values accumulate in FP64, the others in FP32.
template <int L, typename V, class Src, bool GLOBAL>
__device__ __forceinline__ void row_dot2(const RowPair &rb, const uint16_t *__restrict__ col,
                                         const V *__restrict__ val, int lane, Src src, double &y0, double &y1)
{
    using XT = decltype(src(0));
    constexpr bool D = std::is_same<V, double>::value;
    using AT = typename std::conditional<D, double, float>::type;
    const int a0 = rb.a0, e0 = rb.e0, a1 = rb.a1, e1 = rb.e1;
    AT s0 = 0, s1 = 0;
    const int n0 = e0 - a0, n1 = e1 - a1, nmax = n0 > n1 ? n0 : n1;
    for (int k = lane; k < nmax; k += L * BU) {
        int c0[BU], c1[BU];
        AT v0[BU], v1[BU];
#pragma unroll
        for (int u = 0; u < BU; u++) {
            const int kk = k + u * L;
            const bool in0 = kk < n0, in1 = kk < n1;
            if constexpr (GLOBAL) {
                c0[u] = in0 ? (int)ld_stream(col + a0 + kk) : -1;
                c1[u] = in1 ? (int)ld_stream(col + a1 + kk) : -1;
                v0[u] = in0 ? (AT)ld_stream(val + a0 + kk) : (AT)0;
                v1[u] = in1 ? (AT)ld_stream(val + a1 + kk) : (AT)0;
            } else {  // staged in shared memory
                c0[u] = in0 ? (int)col[a0 + kk] : -1;
                c1[u] = in1 ? (int)col[a1 + kk] : -1;
                v0[u] = in0 ? (AT)val[a0 + kk] : (AT)0;
                v1[u] = in1 ? (AT)val[a1 + kk] : (AT)0;
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
            s0 = vfma(v0[u], (AT)x0[u], s0);
            s1 = vfma(v1[u], (AT)x1[u], s1);
        }
    }
    double d0 = (double)s0, d1 = (double)s1;
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
        d0 += __shfl_xor_sync(0xffffffffu, d0, o, L);
        d1 += __shfl_xor_sync(0xffffffffu, d1, o, L);
    }
    y0 = d0;
    y1 = d1;
}

// One row's sum from a staged pass: lanes stride over the row's entries, BU
// per lane per trip, loaded without predicates -- columns past the row's end
// are read from the stage and masked into the p window (which holds finite
// values: zeros before its first copy), their weights are zero.  Lane sums
// combine in a fixed xor tree.
template <int L, typename V, class Src>
__device__ __forceinline__ double row_dot1_smem(int a, int e, const uint16_t *__restrict__ col,
                                                const V *__restrict__ val, int lane, Src src)
{
    constexpr bool D = std::is_same<V, double>::value;
    using AT = typename std::conditional<D, double, float>::type;
    AT s = 0;
    const int n = e - a;
    for (int k = lane; k < n; k += L * BU) {
#pragma unroll
        for (int u = 0; u < BU; u++) {
            const int kk = k + u * L;
            const int c = (int)col[a + kk] & (PW - 1);
            const AT v = kk < n ? (AT)val[a + kk] : (AT)0;
            s = vfma(v, (AT)src(c), s);
        }
    }
    double d = (double)s;
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o, L);
    return d;
}

// The same for an FP16 pass: one 32-bit word per entry (FP16 value bits in
// the high half, the column offset in the low half), so a slot costs one
// shared-memory load besides its gather.
template <int L, class Src>
__device__ __forceinline__ double row_dot1_cv16(int a, int e, const uint32_t *__restrict__ cv, int lane, Src src)
{
    float s = 0.f;
    const int n = e - a;
    for (int k = lane; k < n; k += L * BU) {
#pragma unroll
        for (int u = 0; u < BU; u++) {
            const int kk = k + u * L;
            const uint32_t w = cv[a + kk];
            const float v = kk < n ? __half2float(__ushort_as_half((unsigned short)(w >> 16))) : 0.f;
            s = fmaf(v, (float)src((int)(w & (uint32_t)(PW - 1))), s);
        }
    }
    double d = (double)s;
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o, L);
    return d;
}

// FP64 row sums of rows i0, i1 (-1: none) of a system over all its panels,
// read from global memory, panels added in order; x in FP64.
template <int L>
__device__ __forceinline__ void row_dot2_fp64_all(const BatchArgs &a, const SysView &v, const double *xs, int i0,
                                                  int i1, int lane, double &y0, double &y1)
{
    y0 = 0.0;
    y1 = 0.0;
    for (int k = 0; k < v.npan; k++) {
        const long long rpb = a.prow0[v.gp0 + k], eb = a.pent0[v.gp0 + k];
        const int *rp = a.prow + rpb;
        RowPair rr;
        rr.a0 = i0 >= 0 ? rp[i0] : 0;
        rr.e0 = i0 >= 0 ? rp[i0 + 1] : 0;
        rr.a1 = i1 >= 0 ? rp[i1] : 0;
        rr.e1 = i1 >= 0 ? rp[i1 + 1] : 0;
        const double *xk = xs + (long long)k * PW;
        auto src = [=](int c) -> double { return xk[c]; };
        double t0, t1;
        row_dot2<L, double, decltype(src), true>(rr, a.col + eb, a.val + eb, lane, src, t0, t1);
        y0 += t0;
        y1 += t1;
    }
}

// ---- chunk classes ----------------------------------------------------------

__device__ __forceinline__ float slog10(float v) { return log10f(fmaxf(v, 1e-30f)); }

// The reference's thresholds on a chunk's largest |p_new - p_old| (FP64),
// mapped to the classes a row chunk can run in.
__device__ __forceinline__ int rule_chunk_class(double v, int stat)
{
    if (stat & 1) return 1;          // exact in FP16
    if (!(stat & 2)) return 0;       // FP16 scales out of range
    return v > 1e-6 ? 0 : 1;         // FP64 / FP32 decisions -> FP32; FP16 / INT8 / BYPASS -> FP16
}

// Checkpoint statistics of chunk c (rows [r0, r1) of a system): maxima of
// |r|, |p_new|, |p_new - p_old|, |q| by one warp, written to cdyn[c][0..3];
// with `label`, also the FP16 perturbation ratio ||dq|| / ||q|| of the
// chunk's rows (dq = A16 p - A p over the off-diagonal entries, in FP64),
// written to cdyn[c][8].  Lane results combine in a fixed tree.
template <typename VT>
__device__ void chunk_stats_warp(const BatchArgs &a, const SysView &v, int c, int r0, int r1, const VT *r,
                                 const VT *pn, const VT *po, const VT *q, const float *rscale, bool label, float &gr,
                                 float &gp)
{
    const int lane = threadIdx.x & 31;
    float mr = 0.f, mp = 0.f, mdp = 0.f, mq = 0.f;
    double num = 0.0, den = 0.0;
    for (int i = r0 + lane; i < r1; i += 32) {
        const double pv = (double)pn[i];
        mr = fmaxf(mr, (float)fabs((double)r[i]));
        mp = fmaxf(mp, (float)fabs(pv));
        mdp = fmaxf(mdp, (float)fabs(pv - (double)po[i]));
        mq = fmaxf(mq, (float)fabs((double)__ldcg(q + i)));
        if (label) {
            const double s = (double)rscale[i];
            double dq = 0.0, qq = 0.0;
            for (int k = 0; k < v.npan; k++) {
                const long long rpb = a.prow0[v.gp0 + k], eb = a.pent0[v.gp0 + k];
                for (int e = a.prow[rpb + i]; e < a.prow[rpb + i + 1]; e++) {
                    const int j = (int)a.col[eb + e] + k * PW;
                    const double pj = (double)pn[j], av = a.val[eb + e];
                    qq = fma(av, pj, qq);
                    if (j != i) dq = fma((double)__half2float(a.val16[eb + e]) * s - av, pj, dq);
                }
            }
            num = fma(dq, dq, num);
            den = fma(qq, qq, den);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mp = fmaxf(mp, __shfl_xor_sync(0xffffffffu, mp, o));
        mdp = fmaxf(mdp, __shfl_xor_sync(0xffffffffu, mdp, o));
        mq = fmaxf(mq, __shfl_xor_sync(0xffffffffu, mq, o));
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    if (lane == 0) {
        float *d = a.cdyn + (size_t)c * NCDYN;
        d[0] = mr;
        d[1] = mp;
        d[2] = mdp;
        d[3] = mq;
        if (label) d[8] = den > 0.0 ? (float)(sqrt(num) / sqrt(den)) : (num > 0.0 ? 1e30f : 0.f);
    }
    gr = fmaxf(gr, mr);
    gp = fmaxf(gp, mp);
}

// The 16 features of chunk c (lane 0 writes them to x):
//   0-4 static: log10 max|a| / 10, log10 min|a| / 10, entries / 2048,
//       log10 max_i (S_i / m_i) / 10 (S_i the row's off-diagonal |a| sum,
//       m_i = a_ii - S_i its diagonal-dominance margin), log10 of the largest
//       off-diagonal dynamic range of a row / 10
//   5   log10(||r|| / ||b||) / 10
//   6   log10(max_c |r| / max |r|) / 10      7  log10(max_c |p| / max |p|) / 10
//   8   log10(max_c |dp| / max_c |p|) / 10   9  log10(max_c |q| / (max_c |p| max_c |a|)) / 10
//  10-13 features 6-9 at the previous checkpoint (the current ones at the first)
//  14  reliable updates so far / 16          15 1
__device__ __forceinline__ void chunk_features(const BatchArgs &a, int c, float relres, float gr, float gp, int refs,
                                               bool have_prev, float *x)
{
    const float *s = a.cstat + (size_t)c * NCSTAT;
    float *d = a.cdyn + (size_t)c * NCDYN;
    for (int k = 0; k < 5; k++) x[k] = s[k];
    x[5] = slog10(relres) * 0.1f;
    const float amax = s[5];
    x[6] = slog10(gr > 0.f ? d[0] / gr : 0.f) * 0.1f;
    x[7] = slog10(gp > 0.f ? d[1] / gp : 0.f) * 0.1f;
    x[8] = slog10(d[1] > 0.f ? d[2] / d[1] : 0.f) * 0.1f;
    x[9] = slog10(d[1] > 0.f && amax > 0.f ? d[3] / (d[1] * amax) : 0.f) * 0.1f;
    for (int k = 0; k < 4; k++) x[10 + k] = have_prev ? d[4 + k] : x[6 + k];
    x[14] = (float)refs * (1.f / 16.f);
    x[15] = 1.f;
}

// The policy's class for one chunk: one warp evaluates the network (lane j
// holds hidden unit j), in the same operation order as the host-launched
// classifier.  1 = FP16 when P(label <= FP16) >= LEARN_CONF.
__device__ __forceinline__ int learned_chunk_class(const float *w, const float *x, int stat)
{
    float o[PN_NO];
    pn_forward_warp(w, x, o);
    if (stat & 1) return 1;
    if (!(stat & 2)) return 0;
    float mx = o[0];
    for (int k = 1; k < PN_NO; k++) mx = fmaxf(mx, o[k]);
    float e[PN_NO], z = 0.f;
    for (int k = 0; k < PN_NO; k++) {
        e[k] = expf(o[k] - mx);
        z += e[k];
    }
    return (e[0] + e[1] >= LEARN_CONF * z) ? 1 : 0;
}

// Thread 0: copy panel `k` of p (FP32: p[k PW .. min(n, (k+1) PW))) into the
// shared-memory window; shift_elems receives the position of p[k PW] in the
// window (the copy starts at the 16-byte boundary below it).
__device__ __forceinline__ void issue_pwin(uint64_t *bar, unsigned char *win, const float *p, int n, int k,
                                           int &shift_elems)
{
    const long long a0 = (long long)k * PW, a1 = min((long long)n, a0 + PW);
    const unsigned long long base = (unsigned long long)(p + a0);
    const unsigned long long c0 = base & ~15ull, c1 = ((unsigned long long)(p + a1) + 15ull) & ~15ull;
    shift_elems = (int)((base - c0) >> 2);
    // p was written by the cluster's threads (generic proxy) before the
    // cluster barrier; the bulk copy reads it through the async proxy
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, (unsigned)(c1 - c0));
    bulk_g2s(win, (const void *)c0, (unsigned)(c1 - c0), bar);
}

#ifndef MF_BATCH_MINB
#define MF_BATCH_MINB 1
#endif

template <int L, bool MIX>
__global__ void __launch_bounds__(BNT, MF_BATCH_MINB) k_batched_cg(BatchArgs a)
{
    using VT = typename std::conditional<MIX, float, double>::type;
    using SG = Stage<MIX>;
    using SL = SmemLayout<MIX>;
    constexpr int NS = SG::NS;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double s_warp[BNW];
    __shared__ double s_slot[8];
    __shared__ float s_fslot[2];
    __shared__ float s_fwarp[2 * BNW];
    __shared__ int s_sys;
    __shared__ int s_fail;
    __shared__ int s_pshift;
    extern __shared__ __align__(16) unsigned char b_smem_raw[];
    BSmem<MIX> &S = *reinterpret_cast<BSmem<MIX> *>(b_smem_raw);
    unsigned char *s_win = b_smem_raw + SL::PWIN;
    float *s_w = reinterpret_cast<float *>(b_smem_raw + SL::W);
    float *s_feat = reinterpret_cast<float *>(b_smem_raw + SL::FEAT);
    const bool learned = MIX && a.policy == MF_POLICY_LEARNED && a.mlp_w;
    const bool rule = MIX && a.policy == MF_POLICY_RULE;
    const bool collect = !MIX && a.collect_every > 0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; k++) {
            mbar_init(&S.bar[k], 1);
            mbar_init(&S.empty[k], MIX ? (BNW - 1) / MF_BATCH_GROUPS : BNW - 1);  // the stage's consumer warps
        }
        mbar_init(&S.pbar, 1);
        mbar_init(&S.wempty, BNW - 1);
        mbar_fence_init();
    }
    if (learned)
        for (int k = threadIdx.x; k < PN_NPARAM; k += BNT) s_w[k] = __bfloat162float(a.mlp_w[k]);
    // the p window holds finite values from the start (padded slots of the
    // row loop read it with zero weight)
    if (MIX)
        for (int k = threadIdx.x; k < (int)(SL::PWIN_BYTES / 4); k += BNT) ((float *)s_win)[k] = 0.f;
    __syncthreads();
    // mbarrier phase parities, one bit per stage (registers: an array indexed
    // by the stage number would live in local memory).  Producer (thread 0):
    // fills of each stage and of the window so far (parity), which stages /
    // whether the window were filled at all.  Consumers: passes consumed per
    // stage and windows consumed (parity).
    unsigned pfill = 0, pstarted = 0, wpar = 0, wstarted = 0;
    unsigned cfull = 0, cwpar = 0;
    const unsigned rank = cl.block_rank(), ncta = cl.num_blocks();
    const int tid = threadIdx.x;
    const int lane = tid % L, grp = tid / L;
    const int wid = tid >> 5, wl = tid & 31;
    constexpr int GPB = BNT / L;  // row groups per CTA
    for (;;) {
        // after a wait that gave up (status word set) no cluster takes another
        // system: the stages' barrier phases of the failed CTA are not known
        if (rank == 0 && tid == 0) s_sys = ld_volatile_i32(a.queue + 1) != 0 ? a.count : atomicAdd(a.queue, 1);
        cl.sync();
        const int qi = *cl.map_shared_rank(&s_sys, 0);
        cl.sync();  // every CTA has read the index before rank 0 writes the next
        if (qi >= a.count) break;
        const int sys = a.order[qi];
        const SysView V = sys_view(a, sys);
        const long long r0 = V.r0;
        const double *b = a.b + r0;
        double *x = a.x + r0;
        const float *rscale = a.rscale + r0;
        VT *r = (VT *)a.r + r0, *q = (VT *)a.q + r0, *xlo = (VT *)a.xlo + r0;
        VT *pb[2] = {(VT *)a.p0 + r0, (VT *)a.p1 + r0};
        // this CTA's chunks and rows
        const int sc0 = a.sc[sys], nch = a.sc[sys + 1] - sc0;
        const int cl0 = sc0 + (int)((long long)nch * rank / ncta), cl1 = sc0 + (int)((long long)nch * (rank + 1) / ncta);
        const int nchl = cl1 - cl0;
        const int ra = a.crow[cl0 + sys], rb = a.crow[cl1 + sys];
        const int npan = V.npan;
        const int J = nchl * npan;  // (chunk, panel) passes per SpMV, panel-major
        unsigned long long st_bytes = 0, st_lowp = 0, st_pass = 0;  // thread 0: passes issued
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
        if (MIX)
            for (int c = cl0 + tid; c < cl1; c += BNT) a.ccls[c] = (a.ccls_static[c] & 1) ? 1 : 0;
        const double bb = cluster_sum(cl, lb, &s_slot[0], s_warp);
        double rho = MIX ? cluster_sum(cl, lr, &s_slot[1], s_warp) : bb;
        const double nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
        double beta = 0.0, rmax = sqrt(rho), relres = sqrt(rho) / nb;
        int it = 0, refs = 0, status = MF_OK;
        bool lowp_off = false, have_prev = false;
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
            // SpMV needs all of p.  RULE: one warp per chunk, deciding the
            // chunk's class from its own rows' change.
            if (rule && !lowp_off) {
                for (int c = cl0 + wid; c < cl1; c += BNW) {
                    const int c0 = a.crow[c + sys], c1 = a.crow[c + 1 + sys];
                    double v = 0.0;
                    for (int i = c0 + wl; i < c1; i += 32) {
                        const VT pv = vfma(bt, pold[i], r[i]);
                        pnew[i] = pv;
                        if (npan == 2) q[i] = (VT)0;
                        v = fmax(v, fabs((double)pv - (double)pold[i]));
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
                    if (wl == 0) a.ccls[c] = (unsigned char)rule_chunk_class(v, a.ccls_static[c]);
                }
            } else {
                // four rows per thread in flight: loads first, then the stores
                int i = ra + tid;
                for (; i + 3 * BNT < rb; i += 4 * BNT) {
                    VT po4[4], r4[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        po4[u] = pold[i + u * BNT];
                        r4[u] = r[i + u * BNT];
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        pnew[i + u * BNT] = vfma(bt, po4[u], r4[u]);
                        if (npan == 2) q[i + u * BNT] = (VT)0;
                    }
                }
                for (; i < rb; i += BNT) {
                    pnew[i] = vfma(bt, pold[i], r[i]);
                    if (npan == 2) q[i] = (VT)0;
                }
            }
            cl.sync();
            double loc = 0.0;
            // SpMV.  Warp 0 produces: its lanes load the descriptors of 32
            // (chunk, panel) passes at a time and lane 0 issues their bulk
            // copies into NS shared-memory stages, each stage refilled once
            // the consumers have released it (empty barrier), and before the
            // first pass of each panel the copy of p's window for that panel
            // (mixed kernel) once the previous window is released.  Warps
            // 1.. consume: wait for a stage (full barrier), compute its rows,
            // release it -- no CTA-wide barrier per pass.  Every wait is
            // bounded; a failure is voted CTA-wide and cluster-wide below.
            bool fail = false;
            if (J > 0) {
                if (wid == 0) {
                    // descriptors of the next 32 passes load while the current
                    // ones are issued
                    BChunk dn;
                    memset(&dn, 0, sizeof(dn));
                    if (wl < J) dn = b_chunk(a, sys, V, cl0 + wl % nchl, wl / nchl, MIX);
                    for (int jb = 0; jb < J && !fail; jb += 32) {
                        const BChunk d = dn;
                        memset(&dn, 0, sizeof(dn));
                        if (jb + 32 + wl < J)
                            dn = b_chunk(a, sys, V, cl0 + (jb + 32 + wl) % nchl, (jb + 32 + wl) / nchl, MIX);
                        const int cnt = min(32, J - jb);
                        for (int t = 0; t < cnt; t++) {
                            BChunk ch;
                            ch.r0 = __shfl_sync(0xffffffffu, d.r0, t);
                            ch.r1 = __shfl_sync(0xffffffffu, d.r1, t);
                            ch.e0 = __shfl_sync(0xffffffffu, d.e0, t);
                            ch.e1 = __shfl_sync(0xffffffffu, d.e1, t);
                            ch.cls = __shfl_sync(0xffffffffu, d.cls, t);
                            ch.panel = __shfl_sync(0xffffffffu, d.panel, t);
                            ch.ebase = __shfl_sync(0xffffffffu, d.ebase, t);
                            ch.rpbase = __shfl_sync(0xffffffffu, d.rpbase, t);
                            ch.rowbase = __shfl_sync(0xffffffffu, d.rowbase, t);
                            const int j = jb + t, k = j % NS;
                            int ok = 1;
                            if (wl == 0) {
                                if (MIX && j % nchl == 0) {
                                    if (wstarted)
                                        ok = mbar_wait_sleep_bounded(&S.wempty, wpar ^ 1u, a.queue + 1, a.budget_ns,
                                                                     a.backoff_ns);
                                    if (ok) {
                                        issue_pwin(&S.pbar, s_win, (const float *)pnew, V.n, j / nchl, s_pshift);
                                        wpar ^= 1u;
                                        wstarted = 1;
                                    }
                                }
                                if (ok && ((pstarted >> k) & 1u))
                                    ok = mbar_wait_sleep_bounded(&S.empty[k], ((pfill >> k) & 1u) ^ 1u, a.queue + 1,
                                                           a.budget_ns, a.backoff_ns);
                                if (ok) {
                                    b_issue<MIX>(a, S, ch, k);
                                    pfill ^= 1u << k;
                                    pstarted |= 1u << k;
                                    st_bytes += chunk_bytes<MIX>(ch);
                                    st_lowp += ch.cls;
                                    st_pass++;
                                }
                            }
                            ok = __shfl_sync(0xffffffffu, ok, 0);
                            if (!ok) {
                                fail = true;
                                break;
                            }
                        }
                    }
                } else {
                    // consumer warps in NGRP groups: group g consumes the
                    // passes j with j % NGRP == g (stages j % NS, two per
                    // group), its CWS warps splitting each pass's rows;
                    // every consumer warp waits for each panel's window and
                    // releases it after its own passes of that panel
                    // (mixed kernel; the FP64 kernel's consumer warps all
                    // take every pass, so that a row's panels are added in
                    // panel order without a window to order them)
                    constexpr int NCW = BNW - 1;
                    constexpr int NGRP = MIX ? MF_BATCH_GROUPS : 1;
                    constexpr int CWS = NCW / NGRP;             // consumer warps per group
                    static_assert(NCW % NGRP == 0 && NS % NGRP == 0, "groups split the warps and stages evenly");
                    const int cw = wid - 1;
                    const int kg = cw / CWS;                    // this warp's group
                    const int gr = cw % CWS;                    // warp within the stage's group
                    const int ct = gr * 32 + wl;                // thread within the stage's group
                    const int clane = ct % L, cgrp = ct / L;
                    constexpr int GPC = CWS * 32 / L;           // row groups per stage
                    const int nwin = MIX ? npan : 1;
                    for (int pw = 0; pw < nwin && !fail; pw++) {
                        const int j0 = MIX ? pw * nchl : 0, j1 = MIX ? j0 + nchl : J;
                        if (MIX) {
                            const bool ww =
                                mbar_wait_sleep_bounded(&S.pbar, cwpar, a.queue + 1, a.budget_ns, a.backoff_ns);
                            cwpar ^= 1u;
                            if (!__all_sync(0xffffffffu, ww)) {
                                fail = true;
                                break;
                            }
                        }
                        const int jfirst = j0 + (kg - j0 % NGRP + NGRP) % NGRP;
                        for (int j = jfirst; j < j1; j += NGRP) {
                            const int k = j % NS;
                            bool w = mbar_wait_sleep_bounded(&S.bar[k], (cfull >> k) & 1u, a.queue + 1, a.budget_ns,
                                                             a.backoff_ns);
                            cfull ^= 1u << k;
                            if (!__all_sync(0xffffffffu, w)) {
                                fail = true;
                                break;
                            }
                            const BHdr &h = S.hdr[k];
                            const unsigned char *st = S.stage[k];
                            const int *rps = (const int *)(st + SG::OFF_RP + h.sh_rp);  // panel row pointers of h.r0 ..
                            const int nr = h.r1 - h.r0;
                            const bool h16 = MIX && h.cls == 1;
                            const bool firstp = h.panel == 0;
                            const VT *pwin = MIX ? (const VT *)s_win + s_pshift : (const VT *)pnew + (long long)h.panel * PW;
                            auto psrc = [=](int c) -> VT { return pwin[c]; };
                            const uint16_t *scol = (const uint16_t *)(st + SG::OFF_COL + h.sh_col);
                            const unsigned char *sval = st + SG::OFF_VAL + h.sh_val;
                            // the row sum of row q0 of this pass goes to q (FP16
                            // rows: scaled, plus the FP32 diagonal times the
                            // diagonal's p from the window of the panel that
                            // holds the diagonal column).  One panel: the row
                            // sum is q; two panels: both partial sums are added
                            // to q (zeroed by the p update; two additions onto
                            // zero give the same bits in either order); more
                            // panels: added in panel order (the mixed kernel's
                            // window barrier orders the panels; the FP64
                            // kernel's warps take every pass in order).
                            auto row_out = [&](int q0, double y0) {
                                const int i0 = h.r0 + q0;
                                if (h16) {
                                    const float *srs = (const float *)(st + SG::OFF_RS + h.sh_rs);
                                    const float *sdg = (const float *)(st + SG::OFF_DG + h.sh_dg);
                                    const float dt =
                                        (i0 / PW == h.panel) ? sdg[q0] * (float)pwin[i0 - h.panel * PW] : 0.f;
                                    y0 = (double)fmaf(srs[q0], (float)y0, dt);
                                }
                                VT *qi = q + i0;
                                if (npan == 1) *qi = (VT)y0;
                                else if (npan == 2) atomicAdd(qi, (VT)y0);
                                else *qi = firstp ? (VT)y0 : (VT)((double)*qi + y0);
                            };
                            if (MIX && !h.direct && a.rowsum == 0) {
                                // two phases over this warp's share of the
                                // pass's rows: (1) the products of its entries,
                                // consecutive entries to consecutive lanes,
                                // written over the staged values in place;
                                // (2) one lane per row adds its products in
                                // entry order
                                const int qa = (int)((long long)nr * gr / CWS);
                                const int qe = (int)((long long)nr * (gr + 1) / CWS);
                                uint32_t *pv = (uint32_t *)(st + SG::OFF_VAL + h.sh_val);
                                if (qa < qe) {
                                    const int ea = rps[qa] - h.e0, eb = rps[qe] - h.e0;
                                    if (h16) {
                                        MF_UNROLL(MF_BATCH_P1U)
                                        for (int e = ea + wl; e < eb; e += 32) {
                                            const uint32_t wv = pv[e];
                                            const float v = __half2float(__ushort_as_half((unsigned short)(wv >> 16)));
                                            pv[e] = __float_as_uint(v * (float)pwin[wv & (uint32_t)(PW - 1)]);
                                        }
                                    } else {
                                        MF_UNROLL(MF_BATCH_P1U)
                                        for (int e = ea + wl; e < eb; e += 32)
                                            pv[e] = __float_as_uint(__uint_as_float(pv[e]) * (float)pwin[scol[e]]);
                                    }
                                    __syncwarp();
                                    for (int q0 = qa + wl; q0 < qe; q0 += 32) {
                                        const int s0 = rps[q0] - h.e0, s1 = rps[q0 + 1] - h.e0;
                                        float acc = 0.f;
                                        for (int e = s0; e < s1; e++) acc += __uint_as_float(pv[e]);
                                        row_out(q0, (double)acc);
                                    }
                                }
                                // the products written here precede the next
                                // bulk copy into this stage
                                fence_proxy_async_smem();
                            } else
                            // one row per lane group; the trip count is the same
                            // for every lane of a warp (shuffles inside)
                            for (int qb = 0; qb < nr; qb += GPC) {
                                const int q0 = qb + cgrp;
                                const bool in = q0 < nr;
                                const int ra0 = in ? rps[q0] : 0, re0 = in ? rps[q0 + 1] : 0;
                                double y0;
                                if (h.direct) {
                                    RowPair rr{ra0, re0, 0, 0};
                                    const uint16_t *gcol = a.col + h.ebase;
                                    double y1;
                                    if constexpr (MIX) {
                                        if (h16)
                                            row_dot2<L, __half, decltype(psrc), true>(rr, gcol, a.val16 + h.ebase, clane,
                                                                                       psrc, y0, y1);
                                        else
                                            row_dot2<L, float, decltype(psrc), true>(rr, gcol, a.val32 + h.ebase, clane,
                                                                                      psrc, y0, y1);
                                    } else {
                                        row_dot2<L, double, decltype(psrc), true>(rr, gcol, a.val + h.ebase, clane, psrc,
                                                                                   y0, y1);
                                    }
                                } else if constexpr (MIX) {
                                    if (h16)
                                        y0 = row_dot1_cv16<L>(ra0 - h.e0, re0 - h.e0, (const uint32_t *)sval, clane, psrc);
                                    else
                                        y0 = row_dot1_smem<L, float>(ra0 - h.e0, re0 - h.e0, scol, (const float *)sval,
                                                                     clane, psrc);
                                } else {
                                    y0 = row_dot1_smem<L, double>(ra0 - h.e0, re0 - h.e0, scol, (const double *)sval,
                                                                  clane, psrc);
                                }
                                if (clane == 0 && in) row_out(q0, y0);
                            }
                            __syncwarp();
                            if (wl == 0) mbar_arrive(&S.empty[k]);
                        }
                        if (fail) break;
                        if (MIX) {
                            __syncwarp();
                            if (wl == 0) mbar_arrive(&S.wempty);
                        }
                    }
                }
            }
            // CTA-wide vote; on a failure the producing thread waits (bounded)
            // for the copies it issued that may still be landing
            fail = __syncthreads_or(fail) != 0;
            if (fail && tid == 0) {
                for (int k = 0; k < NS; k++)
                    if ((pstarted >> k) & 1u) mbar_drain(&S.bar[k], ((pfill >> k) & 1u) ^ 1u, a.queue + 1, a.budget_ns);
                if (MIX && wstarted) mbar_drain(&S.pbar, wpar ^ 1u, a.queue + 1, a.budget_ns);
            }
            if (tid == 0) s_fail = fail ? 1 : 0;
            // p.q over this CTA's rows (q read past L1: partial sums arrive by
            // reductions in L2)
            if (!fail) {
                int i = ra + tid;
                for (; i + 3 * BNT < rb; i += 4 * BNT) {
                    VT p4[4], q4[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        p4[u] = pnew[i + u * BNT];
                        q4[u] = __ldcg(q + i + u * BNT);
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) loc += (double)p4[u] * (double)q4[u];
                }
                for (; i < rb; i += BNT) loc += (double)pnew[i] * (double)__ldcg(q + i);
            }
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
            {
                // four rows per thread in flight (loads first)
                int i = ra + tid;
                for (; i + 3 * BNT < rb; i += 4 * BNT) {
                    VT p4[4], q4[4], r4[4];
                    double x4[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        p4[u] = pnew[i + u * BNT];
                        q4[u] = __ldcg(q + i + u * BNT);
                        r4[u] = r[i + u * BNT];
                        x4[u] = MIX ? (double)xlo[i + u * BNT] : x[i + u * BNT];
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if (MIX) {
                            xlo[i + u * BNT] = fmaf((float)alpha, (float)p4[u], (float)x4[u]);
                            const float ri = fmaf(-(float)alpha, (float)q4[u], (float)r4[u]);
                            r[i + u * BNT] = ri;
                            loc += (double)ri * (double)ri;
                        } else {
                            x[i + u * BNT] = fma(alpha, (double)p4[u], x4[u]);
                            const double ri = fma(-alpha, (double)q4[u], (double)r4[u]);
                            r[i + u * BNT] = ri;
                            loc += ri * ri;
                        }
                    }
                }
                for (; i < rb; i += BNT) {
                    if (MIX) {
                        xlo[i] = fmaf((float)alpha, (float)pnew[i], (float)xlo[i]);
                        const float ri = fmaf(-(float)alpha, (float)__ldcg(q + i), (float)r[i]);
                        r[i] = ri;
                        loc += (double)ri * (double)ri;
                    } else {
                        x[i] = fma(alpha, (double)pnew[i], x[i]);
                        const double ri = fma(-alpha, (double)__ldcg(q + i), (double)r[i]);
                        r[i] = ri;
                        loc += ri * ri;
                    }
                }
            }
            double rho_new = cluster_sum(cl, loc, &s_slot[3], s_warp);
            it++;
            bool checkpoint = learned && !lowp_off && it == 1;
            if (MIX && (sqrt(rho_new) <= a.delta * rmax || sqrt(rho_new) <= a.tol * nb)) {
                for (int i = ra + tid; i < rb; i += BNT) {
                    x[i] += (double)xlo[i];
                    xlo[i] = (VT)0;
                }
                cl.sync();
                loc = 0.0;
                for (int base = ra; base < rb; base += 2 * GPB) {
                    const int i0 = base + grp < rb ? base + grp : -1;
                    const int i1 = base + GPB + grp < rb ? base + GPB + grp : -1;
                    double y0, y1;
                    row_dot2_fp64_all<L>(a, V, x, i0, i1, lane, y0, y1);
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
                const double rt = sqrt(rho_new);
                // the low-precision classes stop where the FP64 residual did
                // not follow the recurrence (uniform: every CTA holds the same
                // cluster sums)
                if ((rule || learned) && !lowp_off && rt > 0.5 * rmax) {
                    lowp_off = true;
                    for (int c = cl0 + tid; c < cl1; c += BNT) a.ccls[c] = (a.ccls_static[c] & 1) ? 1 : 0;
                }
                rmax = rt;
                refs++;
                checkpoint = learned && !lowp_off;
            }
            const bool sample = collect && (it % a.collect_every == 1 || a.collect_every == 1);
            if (checkpoint || sample) {
                // checkpoint statistics: one warp per chunk of this CTA, then
                // the system's maxima of |r| and |p| over the cluster
                float gr = 0.f, gp = 0.f;
                for (int c = cl0 + wid; c < cl1; c += BNW)
                    chunk_stats_warp<VT>(a, V, c, a.crow[c + sys], a.crow[c + 1 + sys], r, pnew, pold, q, rscale,
                                         sample, gr, gp);
                cluster_max2(cl, gr, gp, s_fslot, s_fwarp);
                const float rel = (float)(sqrt(rho_new) / nb);
                float *xf = s_feat + wid * PN_NF;
                for (int c = cl0 + wid; c < cl1; c += BNW) {
                    if (wl == 0) chunk_features(a, c, rel, gr, gp, refs, have_prev, xf);
                    __syncwarp();
                    float *d = a.cdyn + (size_t)c * NCDYN;
                    if (checkpoint) {
                        const int cls = learned_chunk_class(s_w, xf, a.ccls_static[c]);
                        if (wl == 0) a.ccls[c] = (unsigned char)cls;
                    } else if (wl == 0) {
                        const unsigned h = ((unsigned)c * 2654435761u) ^ (a.collect_salt + (unsigned)it * 0x9E3779B9u);
                        if ((h >> 8) % (unsigned)a.collect_stride == 0u) {
                            const unsigned long long slot = atomicAdd(a.ccount, 1ull);
                            if ((long long)slot < a.ccap) {
                                for (int k = 0; k < PN_NF; k++) a.cx[slot * PN_NF + k] = xf[k];
                                a.cy[slot] = (unsigned char)((double)d[8] <= LABEL_TAU ? 1 : 2);
                            }
                        }
                    }
                    if (wl == 0)
                        for (int k = 0; k < 4; k++) d[4 + k] = xf[6 + k];
                    __syncwarp();
                }
                have_prev = true;
                __syncthreads();  // classes written before thread 0 issues the next passes
            }
            beta = rho_new / rho;
            rho = rho_new;
            relres = sqrt(rho) / nb;
        }
        if (MIX && status != MF_OK) {
            for (int i = ra + tid; i < rb; i += BNT) x[i] += (double)xlo[i];
        }
        if (tid == 0) {
            atomicAdd(&a.sysstat[3 * sys], st_bytes);
            atomicAdd(&a.sysstat[3 * sys + 1], st_lowp);
            atomicAdd(&a.sysstat[3 * sys + 2], st_pass);
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

// One CTA per system: the LEARNED classes for given FP64 vectors (the
// classifier of the solve, run outside it so that its decisions can be
// checked).  Every chunk of the system is classified.
__global__ void __launch_bounds__(BNT) k_batch_classify(BatchArgs a, const double *r, const double *pn,
                                                        const double *po, const double *q, const double *relres,
                                                        const int *refs, int have_prev, unsigned char *out,
                                                        float *feat_out)
{
    __shared__ float s_w[PN_NPARAM];
    __shared__ float s_feat[BNW * PN_NF];
    __shared__ float s_m[2 * BNW];
    for (int k = threadIdx.x; k < PN_NPARAM; k += BNT) s_w[k] = __bfloat162float(a.mlp_w[k]);
    __syncthreads();
    const int wid = threadIdx.x >> 5, wl = threadIdx.x & 31;
    for (int sys = blockIdx.x; sys < a.count; sys += gridDim.x) {
        const SysView V = sys_view(a, sys);
        const long long r0 = V.r0;
        const int sc0 = a.sc[sys], sc1 = a.sc[sys + 1];
        float gr = 0.f, gp = 0.f;
        for (int c = sc0 + wid; c < sc1; c += BNW)
            chunk_stats_warp<double>(a, V, c, a.crow[c + sys], a.crow[c + 1 + sys], r + r0, pn + r0, po + r0, q + r0,
                                     a.rscale + r0, false, gr, gp);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            gr = fmaxf(gr, __shfl_xor_sync(0xffffffffu, gr, o));
            gp = fmaxf(gp, __shfl_xor_sync(0xffffffffu, gp, o));
        }
        __syncthreads();
        if (wl == 0) {
            s_m[2 * wid] = gr;
            s_m[2 * wid + 1] = gp;
        }
        __syncthreads();
        gr = gp = 0.f;
        for (int w = 0; w < BNW; w++) {
            gr = fmaxf(gr, s_m[2 * w]);
            gp = fmaxf(gp, s_m[2 * w + 1]);
        }
        float *xf = s_feat + wid * PN_NF;
        for (int c = sc0 + wid; c < sc1; c += BNW) {
            if (wl == 0) chunk_features(a, c, (float)relres[sys], gr, gp, refs[sys], have_prev != 0, xf);
            __syncwarp();
            const int cls = learned_chunk_class(s_w, xf, a.ccls_static[c]);
            if (wl == 0) {
                out[c] = (unsigned char)cls;
                if (feat_out)
                    for (int k = 0; k < PN_NF; k++) feat_out[(size_t)c * PN_NF + k] = xf[k];
                float *d = a.cdyn + (size_t)c * NCDYN;
                for (int k = 0; k < 4; k++) d[4 + k] = xf[6 + k];
            }
            __syncwarp();
        }
        __syncthreads();
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
    constexpr size_t smem = SmemLayout<MIX>::TOTAL;
    cudaFuncSetAttribute(k_batched_cg<L, MIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batched_cg<L, MIX>, BNT, smem);
    int ctas = sms * (per > 0 ? per : 1);
    ctas = (ctas / cluster) * cluster;
    const int want = count * cluster;
    if (ctas > want) ctas = want;
    if (ctas < cluster) ctas = cluster;
    return ctas;
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
    cfg.dynamicSmemBytes = SmemLayout<MIX>::TOTAL;
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
struct Lanes {
    static int ctas(int lanes, int count, int cluster)
    {
        switch (lanes) {
        case 4: return batched_ctas<4, MIX>(count, cluster);
        case 8: return batched_ctas<8, MIX>(count, cluster);
        case 16: return batched_ctas<16, MIX>(count, cluster);
        default: return batched_ctas<32, MIX>(count, cluster);
        }
    }
    static mf_status launch(int lanes, const BatchArgs &a, int cluster, int ctas, cudaStream_t s)
    {
        switch (lanes) {
        case 4: return launch_batched<4, MIX>(a, cluster, ctas, s);
        case 8: return launch_batched<8, MIX>(a, cluster, ctas, s);
        case 16: return launch_batched<16, MIX>(a, cluster, ctas, s);
        default: return launch_batched<32, MIX>(a, cluster, ctas, s);
        }
    }
};

// One CTA per system: ||b - A x|| / ||b|| in FP64 (panels added in order
// per row).
__global__ void k_batch_resid(BatchArgs a, const double *b, const double *x, double *out)
{
    __shared__ double s_warp[8];
    for (int sys = blockIdx.x; sys < a.count; sys += gridDim.x) {
        const SysView V = sys_view(a, sys);
        double rr = 0.0, bb = 0.0;
        for (int i = threadIdx.x; i < V.n; i += blockDim.x) {
            double y = 0.0;
            for (int k = 0; k < V.npan; k++) {
                const long long rpb = a.prow0[V.gp0 + k], eb = a.pent0[V.gp0 + k];
                double t = 0.0;
                for (int e = a.prow[rpb + i]; e < a.prow[rpb + i + 1]; e++)
                    t += a.val[eb + e] * x[V.r0 + (long long)k * PW + a.col[eb + e]];
                y += t;
            }
            const double d = b[V.r0 + i] - y;
            rr += d * d;
            bb += b[V.r0 + i] * b[V.r0 + i];
        }
        rr = block_sum<256>(rr, s_warp);
        bb = block_sum<256>(bb, s_warp);
        if (threadIdx.x == 0) out[sys] = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
        __syncthreads();
    }
}

// Per row of every system (one CTA per system): the FP32 copy, the
// row-scaled FP16 copy with the diagonal taken out, the row scale and the
// FP32 diagonal, and the row statistics the chunk features use.
// Row scale: 2^(e - 14) with e the exponent of the largest off-diagonal
// magnitude; rows whose scale leaves FP32's normal range, or whose diagonal
// does not fit FP32, are marked not FP16-capable.
__global__ void k_batch_rows(BatchArgs a, float *val32, __half *val16, uint32_t *cv16, float *rscale, float *diag32,
                             float4 *rowstat, unsigned char *rowflag)
{
    for (int sys = blockIdx.x; sys < a.count; sys += gridDim.x) {
        const SysView V = sys_view(a, sys);
        for (int i = threadIdx.x; i < V.n; i += blockDim.x) {
            double offmax = 0.0, offmin = 0.0, S = 0.0, d = 0.0, amin = 0.0;
            for (int k = 0; k < V.npan; k++) {
                const long long rpb = a.prow0[V.gp0 + k], eb = a.pent0[V.gp0 + k];
                for (int e = a.prow[rpb + i]; e < a.prow[rpb + i + 1]; e++) {
                    const double v = a.val[eb + e], av = fabs(v);
                    val32[eb + e] = (float)v;
                    if (av > 0.0 && (amin == 0.0 || av < amin)) amin = av;
                    if ((int)a.col[eb + e] + k * PW == i) {
                        d += v;
                    } else {
                        S += av;
                        if (av > offmax) offmax = av;
                        if (av > 0.0 && (offmin == 0.0 || av < offmin)) offmin = av;
                    }
                }
            }
            const int e = offmax > 0.0 ? ilogb(offmax) - 14 : 0;
            const bool ok = e >= -126 && e <= 127 && isfinite(d) && fabs(d) <= 3.0e38;
            bool exact = ok && (double)(float)d == d;
            for (int k = 0; k < V.npan; k++) {
                const long long rpb = a.prow0[V.gp0 + k], eb = a.pent0[V.gp0 + k];
                for (int q = a.prow[rpb + i]; q < a.prow[rpb + i + 1]; q++) {
                    const double v = a.val[eb + q];
                    __half h = __float2half_rn(0.f);
                    if (ok && (int)a.col[eb + q] + k * PW != i) {
                        h = __double2half(ldexp(v, -e));
                        if ((double)__half2float(h) * ldexp(1.0, e) != v) exact = false;
                    }
                    val16[eb + q] = h;
                    cv16[eb + q] = ((uint32_t)__half_as_ushort(h) << 16) | (uint32_t)a.col[eb + q];
                }
            }
            rscale[V.r0 + i] = ok ? ldexpf(1.f, e) : 0.f;
            diag32[V.r0 + i] = (float)d;
            const double margin = d - S;
            rowstat[V.r0 + i] = make_float4((float)fmax(offmax, fabs(d)), (float)amin,
                                            (float)(S / fmax(margin, 1e-30 * fmax(S, 1e-300))),
                                            offmin > 0.0 ? (float)(offmax / offmin) : 1.f);
            rowflag[V.r0 + i] = (unsigned char)((exact ? 1 : 0) | (ok ? 2 : 0));
        }
    }
}

// Per chunk (one warp per chunk, one CTA per system): the static class byte
// (bit 0 every row exact in FP16, bit 1 every row FP16-capable) and the
// static features.
__global__ void k_batch_chunks(int count, const long long *row0, const int *sc, const int *crow, const int *cent,
                               const float4 *rowstat, const unsigned char *rowflag, unsigned char *ccls_static,
                               float *cstat)
{
    const int wid = threadIdx.x >> 5, wl = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int sys = blockIdx.x; sys < count; sys += gridDim.x) {
        const long long r0 = row0[sys];
        for (int c = sc[sys] + wid; c < sc[sys + 1]; c += nw) {
            const int c0 = crow[c + sys], c1 = crow[c + 1 + sys];
            float amax = 0.f, amin = 3e38f, dd = 0.f, rng = 1.f;
            unsigned flag = 3u;
            for (int i = c0 + wl; i < c1; i += 32) {
                const float4 st = rowstat[r0 + i];
                amax = fmaxf(amax, st.x);
                if (st.y > 0.f) amin = fminf(amin, st.y);
                dd = fmaxf(dd, st.z);
                rng = fmaxf(rng, st.w);
                flag &= rowflag[r0 + i];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
                amin = fminf(amin, __shfl_xor_sync(0xffffffffu, amin, o));
                dd = fmaxf(dd, __shfl_xor_sync(0xffffffffu, dd, o));
                rng = fmaxf(rng, __shfl_xor_sync(0xffffffffu, rng, o));
                flag &= __shfl_xor_sync(0xffffffffu, flag, o);
            }
            if (wl == 0) {
                ccls_static[c] = (unsigned char)flag;
                float *s = cstat + (size_t)c * NCSTAT;
                s[0] = slog10(amax) * 0.1f;
                s[1] = slog10(amin < 3e38f ? amin : 0.f) * 0.1f;
                s[2] = (float)(cent[c + 1 + sys] - cent[c + sys]) * (1.f / 2048.f);
                s[3] = slog10(dd) * 0.1f;
                s[4] = slog10(rng) * 0.1f;
                s[5] = amax;
            }
        }
    }
}

// Host: panel-major storage of one system.  Entries of row i in panel k
// (columns [k PW, (k+1) PW)) keep their order within the row; chunks are
// row ranges of at most BCR rows with at most BCE entries in every panel (a
// row with more is a chunk of its own).
struct HostSys {
    int np = 0;
    std::vector<int> prow;          // np x (n + 1)
    std::vector<long long> pnz;     // entries per panel
    std::vector<uint16_t> col;      // panel-major
    std::vector<double> val;
    std::vector<int> crow, cent;    // chunk row starts (n at the end), scanned entries
};

void host_panels(int n, const int *rp, const int *ci, const double *v, HostSys &h)
{
    const int np = (n + PW - 1) / PW;
    h.np = np;
    h.prow.assign((size_t)np * (n + 1), 0);
    h.pnz.assign(np, 0);
    for (int i = 0; i < n; i++)
        for (int k = rp[i]; k < rp[i + 1]; k++) h.prow[(size_t)(ci[k] / PW) * (n + 1) + i + 1]++;
    long long base = 0;
    std::vector<long long> pbase(np);
    for (int k = 0; k < np; k++) {
        int *p = &h.prow[(size_t)k * (n + 1)];
        for (int i = 0; i < n; i++) p[i + 1] += p[i];
        h.pnz[k] = p[n];
        pbase[k] = base;
        base += p[n];
    }
    h.col.resize((size_t)base);
    h.val.resize((size_t)base);
    std::vector<int> fill((size_t)np);
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < np; k++) fill[k] = h.prow[(size_t)k * (n + 1) + i];
        for (int e = rp[i]; e < rp[i + 1]; e++) {
            const int k = ci[e] / PW;
            const long long at = pbase[k] + fill[k]++;
            h.col[(size_t)at] = (uint16_t)(ci[e] - k * PW);
            h.val[(size_t)at] = v[e];
        }
    }
    // chunks
    h.crow.clear();
    h.cent.clear();
    int r = 0;
    long long ent = 0;
    while (r < n) {
        h.crow.push_back(r);
        h.cent.push_back((int)ent);
        const int r_start = r;
        r++;
        auto fits = [&](int r1) {
            for (int k = 0; k < np; k++) {
                const int *p = &h.prow[(size_t)k * (n + 1)];
                if (p[r1] - p[r_start] > BCE) return false;
            }
            return true;
        };
        while (r < n && r - r_start < BCR && fits(r + 1)) r++;
        ent += rp[r] - rp[r_start];
    }
    h.crow.push_back(n);
    h.cent.push_back((int)ent);
}

}  // namespace
}  // namespace mf

using namespace mf;

namespace {

template <typename F>
void parallel_for(int count, F f)
{
    const int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    std::atomic<int> next{0};
    for (int t = 0; t < nt; t++)
        th.emplace_back([&]() {
            for (int s = next++; s < count; s = next++) f(s);
        });
    for (auto &t : th) t.join();
}

}  // namespace

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
    bt->nz0 = nz0;
    // validation
    for (int s = 0; s < count; s++) {
        for (int i = 0; i < n[s]; i++)
            if (rowptr[s][i + 1] < rowptr[s][i]) {
                delete bt;
                set_last_error("mf_batch_create: system %d row pointers decrease at row %d", s, i);
                return MF_ERR_INVALID_ARG;
            }
        const int e = rowptr[s][n[s]];
        for (int k = 0; k < e; k++) {
            const int c = colidx[s][k];
            if (c < 0 || c >= n[s]) {
                delete bt;
                set_last_error("mf_batch_create: system %d column %d outside [0, %d)", s, c, n[s]);
                return MF_ERR_INVALID_ARG;
            }
        }
    }
    // panel-major storage and chunks of every system (host threads)
    std::vector<HostSys> hs(count);
    parallel_for(count, [&](int s) { host_panels(n[s], rowptr[s], colidx[s], val[s], hs[s]); });
    std::vector<int> pan0(count), npan(count), sc(count + 1), crow, cent;
    std::vector<long long> prow0, pent0;
    long long prows = 0, pents = 0;
    int panels = 0;
    for (int s = 0; s < count; s++) {
        pan0[s] = panels;
        npan[s] = hs[s].np;
        for (int k = 0; k < hs[s].np; k++) {
            prow0.push_back(prows);
            pent0.push_back(pents);
            prows += n[s] + 1;
            pents += hs[s].pnz[k];
        }
        panels += hs[s].np;
        sc[s] = (int)(crow.size() - s);
        crow.insert(crow.end(), hs[s].crow.begin(), hs[s].crow.end());
        cent.insert(cent.end(), hs[s].cent.begin(), hs[s].cent.end());
    }
    prow0.push_back(prows);
    pent0.push_back(pents);
    sc[count] = (int)(crow.size() - count);
    const int nch = sc[count];
    bt->nchunks = nch;
    bt->npanels = panels;
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    auto fail = [&](cudaError_t e) {
        set_last_error("mf_batch_create: %s", cudaGetErrorString(e));
        mf_batch_destroy(bt);
        return e == cudaErrorMemoryAllocation ? MF_ERR_NO_MEMORY : MF_ERR_CUDA;
    };
    float4 *rowstat = nullptr;
    unsigned char *rowflag = nullptr;
    cudaError_t e = cudaSuccess;
#define BT_ALLOC(p, bytes) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    BT_ALLOC(bt->d_order, sizeof(int) * count);
    BT_ALLOC(bt->d_n, sizeof(int) * count);
    BT_ALLOC(bt->d_pan0, sizeof(int) * count);
    BT_ALLOC(bt->d_npan, sizeof(int) * count);
    BT_ALLOC(bt->d_row0, sizeof(long long) * count);
    BT_ALLOC(bt->d_prow0, sizeof(long long) * (panels + 1));
    BT_ALLOC(bt->d_pent0, sizeof(long long) * (panels + 1));
    BT_ALLOC(bt->d_prow, sizeof(int) * (prows + 8));  // slack: 16-byte bulk-copy rounding
    BT_ALLOC(bt->d_sc, sizeof(int) * (count + 1));
    BT_ALLOC(bt->d_crow, sizeof(int) * crow.size());
    BT_ALLOC(bt->d_cent, sizeof(int) * cent.size());
    BT_ALLOC(bt->d_col, sizeof(uint16_t) * (nz + 16));
    BT_ALLOC(bt->d_val, sizeof(double) * (nz + 2));
    BT_ALLOC(bt->d_val32, sizeof(float) * (nz + 4));
    BT_ALLOC(bt->d_val16, sizeof(__half) * (nz + 16));
    BT_ALLOC(bt->d_cv16, sizeof(uint32_t) * (nz + 8));
    BT_ALLOC(bt->d_rscale, sizeof(float) * (rows + 4));
    BT_ALLOC(bt->d_diag32, sizeof(float) * (rows + 4));
    BT_ALLOC(bt->d_ccls, (size_t)nch + 16);
    BT_ALLOC(bt->d_ccls_static, (size_t)nch + 16);
    BT_ALLOC(bt->d_cstat, sizeof(float) * NCSTAT * ((size_t)nch + 1));
    BT_ALLOC(bt->d_cdyn, sizeof(float) * NCDYN * ((size_t)nch + 1));
    BT_ALLOC(bt->d_iters, sizeof(int) * count);
    BT_ALLOC(bt->d_refs, sizeof(int) * count);
    BT_ALLOC(bt->d_status, sizeof(int) * count);
    BT_ALLOC(bt->d_relres, sizeof(double) * count * 2);
    BT_ALLOC(bt->d_sysstat, sizeof(unsigned long long) * 3 * count);
    BT_ALLOC(bt->d_queue, sizeof(int) * 4);
    BT_ALLOC(rowstat, sizeof(float4) * (rows + 1));
    BT_ALLOC(rowflag, (size_t)rows + 16);
#undef BT_ALLOC
#define BT_COPY(dst, src, bytes) \
    if (e == cudaSuccess && (bytes) > 0) e = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice)
    BT_COPY(bt->d_order, order.data(), sizeof(int) * count);
    BT_COPY(bt->d_n, n, sizeof(int) * count);
    BT_COPY(bt->d_pan0, pan0.data(), sizeof(int) * count);
    BT_COPY(bt->d_npan, npan.data(), sizeof(int) * count);
    BT_COPY(bt->d_row0, row0.data(), sizeof(long long) * count);
    BT_COPY(bt->d_prow0, prow0.data(), sizeof(long long) * (panels + 1));
    BT_COPY(bt->d_pent0, pent0.data(), sizeof(long long) * (panels + 1));
    BT_COPY(bt->d_sc, sc.data(), sizeof(int) * (count + 1));
    BT_COPY(bt->d_crow, crow.data(), sizeof(int) * crow.size());
    BT_COPY(bt->d_cent, cent.data(), sizeof(int) * cent.size());
    for (int s = 0; s < count && e == cudaSuccess; s++) {
        const long long pr = prow0[pan0[s]], pe = pent0[pan0[s]];
        BT_COPY(bt->d_prow + pr, hs[s].prow.data(), sizeof(int) * hs[s].prow.size());
        BT_COPY(bt->d_col + pe, hs[s].col.data(), sizeof(uint16_t) * hs[s].col.size());
        BT_COPY(bt->d_val + pe, hs[s].val.data(), sizeof(double) * hs[s].val.size());
    }
#undef BT_COPY
    hs.clear();
    if (e == cudaSuccess) e = cudaMemset(bt->d_cdyn, 0, sizeof(float) * NCDYN * ((size_t)nch + 1));
    if (e == cudaSuccess) {
        const int grid = std::min(count, 1184);
        BatchArgs a;
        memset(&a, 0, sizeof(a));
        a.count = count;
        a.n = bt->d_n;
        a.pan0 = bt->d_pan0;
        a.npan = bt->d_npan;
        a.row0 = bt->d_row0;
        a.prow0 = bt->d_prow0;
        a.pent0 = bt->d_pent0;
        a.prow = bt->d_prow;
        a.col = bt->d_col;
        a.val = bt->d_val;
        k_batch_rows<<<grid, 256>>>(a, bt->d_val32, bt->d_val16, bt->d_cv16, bt->d_rscale, bt->d_diag32, rowstat,
                                    rowflag);
        note_launch();
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            k_batch_chunks<<<grid, 256>>>(count, bt->d_row0, bt->d_sc, bt->d_crow, bt->d_cent, rowstat, rowflag,
                                          bt->d_ccls_static, bt->d_cstat);
            note_launch();
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
        std::vector<unsigned char> st((size_t)nch);
        e = cudaMemcpy(st.data(), bt->d_ccls_static, (size_t)nch, cudaMemcpyDeviceToHost);
        for (unsigned char v : st) {
            bt->static_fp16_chunks += v & 1;
            bt->fp16_allowed_chunks += (v >> 1) & 1;
        }
    }
    if (rowstat) cudaFree(rowstat);
    if (rowflag) cudaFree(rowflag);
    if (e != cudaSuccess) return fail(e);
    *out = bt;
    return MF_OK;
}

mf_status mf_batch_destroy(mf_batch bt)
{
    if (!bt) return MF_OK;
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    void *bufs[] = {bt->d_order,  bt->d_n,      bt->d_pan0,   bt->d_npan,   bt->d_row0,   bt->d_prow0,
                    bt->d_pent0,  bt->d_prow,   bt->d_col,    bt->d_val,    bt->d_val32,  bt->d_val16,
                    bt->d_rscale, bt->d_diag32, bt->d_iters,  bt->d_refs,   bt->d_status, bt->d_relres,
                    bt->d_cv16,
                    bt->work,     bt->d_queue,  bt->d_sc,     bt->d_crow,   bt->d_cent,   bt->d_ccls,
                    bt->d_ccls_static, bt->d_cstat, bt->d_cdyn, bt->d_sysstat};
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

// five vectors of rows_total doubles, each followed by PW + 16 elements of
// slack (the last system's p window copy rounds up to 16 bytes)
static size_t batch_vec_len(mf_batch bt) { return (size_t)bt->rows_total + PW + 16; }

static mf_status batch_work(mf_batch bt)
{
    const size_t need = batch_vec_len(bt) * 8 * 5 + 1024;
    if (bt->work_bytes >= need) return MF_OK;
    if (bt->work) cudaFree(bt->work);
    bt->work = nullptr;
    bt->work_bytes = 0;
    MF_CUDA(cudaMalloc(&bt->work, need));
    MF_CUDA(cudaMemset(bt->work, 0, need));
    bt->work_bytes = need;
    return MF_OK;
}

static BatchArgs batch_args(mf_batch bt, const double *b, double *x, const mf_solve_opts &o)
{
    const size_t rows = batch_vec_len(bt);
    char *w = (char *)bt->work;
    BatchArgs a;
    memset(&a, 0, sizeof(a));
    a.count = bt->count;
    a.order = bt->d_order;
    a.n = bt->d_n;
    a.pan0 = bt->d_pan0;
    a.npan = bt->d_npan;
    a.row0 = bt->d_row0;
    a.prow0 = bt->d_prow0;
    a.pent0 = bt->d_pent0;
    a.prow = bt->d_prow;
    a.col = bt->d_col;
    a.val = bt->d_val;
    a.val32 = bt->d_val32;
    a.val16 = bt->d_val16;
    a.cv16 = bt->d_cv16;
    a.rscale = bt->d_rscale;
    a.diag32 = bt->d_diag32;
    a.b = b;
    a.x = x;
    a.r = w;
    a.p0 = w + rows * 8;
    a.p1 = w + rows * 16;
    a.q = w + rows * 24;
    a.xlo = w + rows * 32;
    a.sc = bt->d_sc;
    a.crow = bt->d_crow;
    a.cent = bt->d_cent;
    a.ccls = bt->d_ccls;
    a.ccls_static = bt->d_ccls_static;
    a.cstat = bt->d_cstat;
    a.cdyn = bt->d_cdyn;
    a.queue = bt->d_queue;
    a.iters = bt->d_iters;
    a.refs = bt->d_refs;
    a.status = bt->d_status;
    a.relres = bt->d_relres;
    a.sysstat = bt->d_sysstat;
    a.maxiter = o.maxiter;
    a.tol = o.tol;
    a.delta = (o.refine_delta > 0 && o.refine_delta < 1) ? o.refine_delta : 0.1;
    a.budget_ns = (unsigned long long)(o.wait_budget_s * 1e9);
    {
        const char *e = getenv("MF_BATCH_BACKOFF_NS");
        a.backoff_ns = e ? (unsigned)atoi(e) : 0u;
        const char *rs = getenv("MF_BATCH_ROWSUM");
        a.rowsum = (rs && !strcmp(rs, "lanes")) ? 1 : 0;
    }
    a.policy = o.policy;
    a.mlp_w = (o.policy == MF_POLICY_LEARNED && bt->policy) ? policy_weights(bt->policy) : nullptr;
    return a;
}

static int batch_ctas(mf_batch bt, bool mixed, int lanes, int cluster)
{
    return mixed ? Lanes<true>::ctas(lanes, bt->count, cluster) : Lanes<false>::ctas(lanes, bt->count, cluster);
}

// Enqueues one batched solve.  Nothing here allocates or queries the device:
// batch_work() and batch_ctas() run before (outside any stream capture).
static mf_status batch_enqueue(mf_batch bt, const BatchArgs &a, bool mixed, int lanes, int cluster, int ctas,
                               cudaStream_t s)
{
    MF_CUDA(cudaMemsetAsync(bt->d_queue, 0, sizeof(int) * 2, s));  // queue head, stage-wait status
    MF_CUDA(cudaMemsetAsync(bt->d_sysstat, 0, sizeof(unsigned long long) * 3 * bt->count, s));
    MF_TRY(mixed ? Lanes<true>::launch(lanes, a, cluster, ctas, s) : Lanes<false>::launch(lanes, a, cluster, ctas, s));
    k_batch_resid<<<std::min(bt->count, 1184), 256, 0, s>>>(a, a.b, a.x, bt->d_relres + bt->count);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

static mf_status batch_check_opts(mf_batch bt, const mf_solve_opts &o)
{
    if (o.tol <= 0 || o.maxiter <= 0 || o.wait_budget_s <= 0) {
        set_last_error("batched CG needs tol > 0, maxiter > 0 and a positive wait budget");
        return MF_ERR_INVALID_ARG;
    }
    if (o.policy < MF_POLICY_FP64 || o.policy > MF_POLICY_STATIC_FP16) {
        set_last_error("batched CG: unknown policy %d", o.policy);
        return MF_ERR_INVALID_ARG;
    }
    if (o.precond) {
        set_last_error("batched CG: no preconditioner");
        return MF_ERR_UNSUPPORTED;
    }
    if (o.policy == MF_POLICY_RULE_SCALED || o.policy == MF_POLICY_STATIC_FP16) {
        set_last_error("batched CG: the scaled rule and STATIC_FP16 are not available (RULE, LEARNED, STATIC, FP64 are;"
                       " its FP16 chunks are row-scaled)");
        return MF_ERR_UNSUPPORTED;
    }
    if (o.policy == MF_POLICY_LEARNED && !bt->policy) {
        set_last_error("batched CG: learned policy requested but none is attached (mf_batch_attach_policy)");
        return MF_ERR_UNSUPPORTED;
    }
    return MF_OK;
}

static void batch_schedule(mf_batch bt, int &lanes, int &cluster)
{
    lanes = bt->tuned_lanes ? bt->tuned_lanes : 4;
    cluster = bt->tuned_cluster ? bt->tuned_cluster : 2;
    if (const char *e = getenv("MF_BATCH_LANES")) lanes = atoi(e);
    if (const char *e = getenv("MF_BATCH_CLUSTER")) cluster = atoi(e);
    if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) lanes = 4;
    if (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16) cluster = 2;
}

mf_status mf_batch_cg_solve(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int use_graph,
                            mf_batch_report *report, void *stream)
{
    if (!bt || !b || !x) return MF_ERR_INVALID_ARG;
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    if (opts) o = *opts;
    MF_TRY(batch_check_opts(bt, o));
    cudaStream_t s = (cudaStream_t)stream;
    int lanes, cluster;
    batch_schedule(bt, lanes, cluster);
    const bool mixed = o.policy != MF_POLICY_FP64;
    MF_TRY(batch_work(bt));
    const int ctas = batch_ctas(bt, mixed, lanes, cluster);
    const BatchArgs a = batch_args(bt, b, x, o);
    cudaEvent_t e0, e1;
    MF_CUDA(cudaEventCreate(&e0));
    MF_CUDA(cudaEventCreate(&e1));
    MF_CUDA(cudaEventRecord(e0, s));
    const int key[7] = {lanes, cluster, o.policy, (int)(o.tol * 1e15), o.maxiter,
                        (int)(a.delta * 1e6), (int)(uintptr_t)a.mlp_w};
    if (use_graph) {
        // one graph per (buffers, configuration): replayed on later calls
        if (!bt->graph || bt->graph_b != b || bt->graph_x != x || memcmp(key, bt->graph_key, sizeof(key))) {
            if (bt->graph) cudaGraphExecDestroy(bt->graph);
            bt->graph = nullptr;
            cudaStream_t cs;
            MF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaGraph_t g;
            MF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            mf_status st = batch_enqueue(bt, a, mixed, lanes, cluster, ctas, cs);
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
        MF_TRY(batch_enqueue(bt, a, mixed, lanes, cluster, ctas, s));
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
    std::vector<unsigned long long> ss((size_t)count * 3);
    MF_CUDA(cudaMemcpy(it.data(), bt->d_iters, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(rf.data(), bt->d_refs, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(stt.data(), bt->d_status, sizeof(int) * count, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(rr.data(), bt->d_relres, sizeof(double) * count * 2, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(ss.data(), bt->d_sysstat, sizeof(unsigned long long) * 3 * count, cudaMemcpyDeviceToHost));
    mf_status worst = MF_OK;
    long long iters = 0, bytes = 0;
    unsigned long long lowp = 0, passes = 0;
    double maxrr = 0;
    int maxit = 0, refs = 0, failed = 0;
    for (int k = 0; k < count; k++) {
        iters += it[k];
        maxit = std::max(maxit, it[k]);
        refs += rf[k];
        maxrr = std::max(maxrr, rr[count + k]);
        lowp += ss[3 * k + 1];
        passes += ss[3 * k + 2];
        // matrix bytes streamed by the (chunk, panel) passes (counted in the
        // kernel), the vector streams of each iteration (p update: r, p_old
        // in, p out; SpMV: p read once, q out; x, r update: p, q, x, r in,
        // x, r out), and per reliable update an FP64 pass over the matrix
        // plus b, x in and r out
        const long long nn = bt->n[k];
        const long long nnz = (k + 1 < count ? bt->nz0[k + 1] : bt->nnz_total) - bt->nz0[k];
        const long long vb = mixed ? 4 : 8;
        bytes += (long long)ss[3 * k] + (long long)it[k] * 11 * vb * nn +
                 (long long)rf[k] * (nnz * (8 + 2) + 4 * (nn + 1) + 16 * nn + vb * nn);
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
        report->bytes_moved = bytes;
        report->fp16_share = passes ? (double)lowp / (double)passes : 0.0;
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

mf_status mf_batch_chunk_count(mf_batch bt, int *chunks, int *static_fp16, int *fp16_capable)
{
    if (!bt) return MF_ERR_INVALID_ARG;
    if (chunks) *chunks = bt->nchunks;
    if (static_fp16) *static_fp16 = bt->static_fp16_chunks;
    if (fp16_capable) *fp16_capable = bt->fp16_allowed_chunks;
    return MF_OK;
}

mf_status mf_batch_export(mf_batch bt, const char *name, void *host_dst, size_t bytes)
{
    if (!bt || !name || (!host_dst && bytes)) return MF_ERR_INVALID_ARG;
    const void *src = nullptr;
    size_t need = 0;
    const size_t nz = (size_t)bt->nnz_total, rows = (size_t)bt->rows_total, nch = (size_t)bt->nchunks;
    if (!strcmp(name, "chunk_class")) src = bt->d_ccls, need = nch;
    else if (!strcmp(name, "chunk_static")) src = bt->d_ccls_static, need = nch;
    else if (!strcmp(name, "chunk_features_static")) src = bt->d_cstat, need = sizeof(float) * NCSTAT * nch;
    else if (!strcmp(name, "chunk_start")) src = bt->d_sc, need = sizeof(int) * (bt->count + 1);
    else if (!strcmp(name, "chunk_rows")) src = bt->d_crow, need = sizeof(int) * (nch + bt->count);
    else if (!strcmp(name, "chunk_ends")) src = bt->d_cent, need = sizeof(int) * (nch + bt->count);
    else if (!strcmp(name, "val16")) src = bt->d_val16, need = 2 * nz;
    else if (!strcmp(name, "val32")) src = bt->d_val32, need = 4 * nz;
    else if (!strcmp(name, "val")) src = bt->d_val, need = 8 * nz;
    else if (!strcmp(name, "col")) src = bt->d_col, need = 2 * nz;
    else if (!strcmp(name, "row_scale")) src = bt->d_rscale, need = 4 * rows;
    else if (!strcmp(name, "diag32")) src = bt->d_diag32, need = 4 * rows;
    else {
        set_last_error("mf_batch_export: unknown array %s", name);
        return MF_ERR_INVALID_ARG;
    }
    if (bytes != need) {
        set_last_error("mf_batch_export: %s has %zu bytes, %zu given", name, need, bytes);
        return MF_ERR_INVALID_ARG;
    }
    if (need) MF_CUDA(cudaMemcpy(host_dst, src, need, cudaMemcpyDeviceToHost));
    return MF_OK;
}

mf_status mf_batch_attach_policy(mf_batch bt, mf_learned p)
{
    if (!bt) return MF_ERR_INVALID_ARG;
    bt->policy = p;
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
    return MF_OK;
}

mf_status mf_batch_policy_classify(mf_batch bt, const double *r, const double *p_new, const double *p_old,
                                   const double *q, const double *relres, const int *refinements, int have_prev,
                                   unsigned char *classes, float *features)
{
    if (!bt || !r || !p_new || !p_old || !q || !relres || !refinements || !classes) return MF_ERR_INVALID_ARG;
    if (!bt->policy) {
        set_last_error("mf_batch_policy_classify: no policy attached");
        return MF_ERR_UNSUPPORTED;
    }
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    o.policy = MF_POLICY_LEARNED;
    BatchArgs a = batch_args(bt, nullptr, nullptr, o);
    k_batch_classify<<<std::min(bt->count, 1184), BNT>>>(a, r, p_new, p_old, q, relres, refinements, have_prev,
                                                         classes, features);
    note_launch();
    MF_CUDA(cudaGetLastError());
    MF_CUDA(cudaDeviceSynchronize());
    return MF_OK;
}

// Plain FP64 batched solve of every system that adds (chunk features,
// label) samples every checkpoint_every iterations (about one chunk in
// sample_stride) to the policy's training set.  Label 1 (FP16) when the
// FP16 values perturb the chunk's A p by at most 2^-6 of it (2-norms over
// the chunk's rows), else 2 (FP32).
mf_status mf_batch_policy_collect(mf_learned p, mf_batch bt, const double *b, int checkpoint_every,
                                  int sample_stride, long long max_samples, long long *samples_out)
{
    if (!p || !bt || !b || checkpoint_every <= 0 || sample_stride <= 0 || max_samples <= 0)
        return MF_ERR_INVALID_ARG;
    float *cx = nullptr;
    unsigned char *cy = nullptr;
    long long have = 0;
    MF_TRY(policy_sample_buffers(p, max_samples, &cx, &cy, &have));
    MF_TRY(batch_work(bt));
    double *x = nullptr;
    unsigned long long *cnt = nullptr;
    MF_CUDA(cudaMalloc(&x, sizeof(double) * (bt->rows_total + 1)));
    MF_CUDA(cudaMalloc(&cnt, sizeof(unsigned long long)));
    const unsigned long long start = (unsigned long long)have;
    MF_CUDA(cudaMemcpy(cnt, &start, sizeof(start), cudaMemcpyHostToDevice));
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    o.policy = MF_POLICY_FP64;
    o.tol = 1e-10;
    o.maxiter = 100000;
    BatchArgs a = batch_args(bt, b, x, o);
    a.collect_every = checkpoint_every;
    a.collect_stride = sample_stride;
    a.collect_salt = (unsigned)(have * 2654435761ull);
    a.cx = cx;
    a.cy = cy;
    a.ccount = cnt;
    a.ccap = max_samples;
    const int lanes = 8, cluster = 2;
    const int ctas = batch_ctas(bt, false, lanes, cluster);
    mf_status st = batch_enqueue(bt, a, false, lanes, cluster, ctas, 0);
    unsigned long long end = start;
    if (st == MF_OK) {
        cudaError_t e = cudaMemcpy(&end, cnt, sizeof(end), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            set_last_error("mf_batch_policy_collect: %s", cudaGetErrorString(e));
            st = MF_ERR_CUDA;
        }
    }
    cudaFree(x);
    cudaFree(cnt);
    if (st != MF_OK) return st;
    const long long total = (long long)std::min<unsigned long long>(end, (unsigned long long)max_samples);
    MF_TRY(policy_sample_commit(p, total));
    if (samples_out) *samples_out = total;
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
    MF_TRY(batch_check_opts(bt, o));
    const int lanes_c[] = {4, 8, 16, 32};
    const int clus_c[] = {1, 2, 4, 8, 16};
    float best = 1e30f;
    int bl = 8, bc = 2;
    cudaStream_t s = (cudaStream_t)stream;
    const bool mixed = o.policy != MF_POLICY_FP64;
    MF_TRY(batch_work(bt));
    const BatchArgs a = batch_args(bt, b, x, o);
    for (int li : lanes_c)
        for (int ci : clus_c) {
            const int ctas = batch_ctas(bt, mixed, li, ci);
            cudaEvent_t e0, e1;
            MF_CUDA(cudaEventCreate(&e0));
            MF_CUDA(cudaEventCreate(&e1));
            MF_CUDA(cudaEventRecord(e0, s));
            mf_status st = batch_enqueue(bt, a, mixed, li, ci, ctas, s);
            MF_CUDA(cudaEventRecord(e1, s));
            MF_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            std::vector<int> stt(bt->count);
            MF_CUDA(cudaMemcpy(stt.data(), bt->d_status, sizeof(int) * bt->count, cudaMemcpyDeviceToHost));
            const bool ok = st == MF_OK && std::all_of(stt.begin(), stt.end(), [](int v) { return v == MF_OK; });
            if (ok && ms < best) {
                best = ms;
                bl = li;
                bc = ci;
            }
        }
    bt->tuned_lanes = bl;
    bt->tuned_cluster = bc;
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
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
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
    return MF_OK;
}

}  // extern "C"
