// multi.cu -- multi-right-hand-side FP64 SpMM and CG (k <= 16 columns).
//
// One pass over the matrix serves every column: the vectors of all k
// systems are stored row-interleaved (entry (i, j) at i * KP + j, KP = k
// rounded up to 4, 8 or 16, padding columns zero), so the gather of one
// matrix entry reads the KP values of its column as one contiguous run.  The
// matrix is read from the row-slot layout (the layout of the persistent FP64
// solver): per 16-row strip, K slots of one entry per row.  A group of KP / 4
// threads shares a row, each thread owning 4 columns; every column's row sum
// is formed in blockspmv_cpu's order (per tile a sequential sum of the row's
// products, tiles added in column order), so column j of A X equals the
// single-vector FP64 SpMV of column j bit for bit.
//
// The CG keeps k independent recurrences (the textbook unpreconditioned CG
// per column: alpha_j = rho_j / p_j.q_j, beta_j = rho_new_j / rho_j) that
// share each SpMM.  Per iteration three launches: the SpMM with the p.q
// partial sums, the x / r update with the r.r partial sums, and p = r + beta
// p.  Per-column sums are deterministic: every block reduces its columns in
// a fixed tree and writes one partial per column; the last block to finish
// (a device-scope counter) adds the partials in block order and updates the
// per-column state.  A converged column keeps alpha = beta = 0 from then on
// (its x and r no longer change); the launches return at once after every
// column has converged or maxiter is reached, so the host queues batches of
// iterations and reads the stop flag between batches.
//
// No tensor cores: FP64 has no tcgen05 kind, and the tiles of the stencil
// systems hold 3-7 entries per row, so a dense-tile MMA would mostly
// multiply zeros.  The gain is the matrix read once for k right-hand sides.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "solver.h"

namespace mf {
namespace {

constexpr int MR_NT = 256;                 // threads per block
constexpr int MR_GRID = 148 * 8;           // fixed grid: the partial sums do not depend on timing
constexpr int MR_MAXK = 16;
constexpr int MR_BATCH = 16;               // iterations queued between stop-flag reads
constexpr int MR_VEC_MINB = 8;             // streaming kernels: 8 blocks per SM (32 registers)
#ifndef MF_MR_SPMM_MINB
#define MF_MR_SPMM_MINB 5
#endif
constexpr int MR_SPMM_MINB = MF_MR_SPMM_MINB;  // SpMM blocks per SM (4: 64 registers, 5: 48)

// Per-solve device state (one struct, zeroed before the solve).
struct MrState {
    double rho[MR_MAXK];     // r.r of the current residual
    double nb[MR_MAXK];      // ||b|| (1 when b is zero)
    double alpha[MR_MAXK];
    double beta[MR_MAXK];
    double rtrue[MR_MAXK];   // ||b - A x|| at exit
    int iters[MR_MAXK];
    int status[MR_MAXK];     // MF_OK, MF_ERR_BREAKDOWN
    int done[MR_MAXK];
    int it;                  // iterations issued
    int stop;                // every column done, or maxiter reached
    unsigned count;          // blocks finished in the current launch (last-block pattern)
};

// Column sums of one block: v is this thread's partial of column tid % KP
// (the vector kernels) -- lanes with the same column are KP apart in a warp.
template <int KP>
__device__ __forceinline__ void block_cols(double v, double (*sw)[MR_MAXK], double *out)
{
    static_assert(32 % KP == 0, "columns repeat every KP lanes");
#pragma unroll
    for (int off = 16; off >= KP; off >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane < KP) sw[w][lane] = v;
    __syncthreads();
    if (threadIdx.x < KP) {
        double s = 0.0;
        for (int i = 0; i < MR_NT / 32; i++) s = __dadd_rn(s, sw[i][threadIdx.x]);
        out[threadIdx.x] = s;
    }
}

// After this block wrote its partials: true in the last block to finish
// (which then sees every block's partials), which also resets the counter.
__device__ __forceinline__ bool mr_last_block(MrState *st)
{
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(&st->count, 1u) == gridDim.x - 1;
        if (last) st->count = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Last block: totals[j] = sum over blocks of partials[b * KP + j], blocks in
// order within MR_NT / KP slices, slices in order.
template <int KP>
__device__ __forceinline__ void sum_partials(const double *partials, double *totals)
{
    constexpr int NS = MR_NT / KP;
    __shared__ double s_sl[MR_NT];
    const int j = threadIdx.x % KP, q = threadIdx.x / KP;
    const int G = gridDim.x, per = (G + NS - 1) / NS;
    const int b0 = q * per, b1 = min(G, b0 + per);
    double s = 0.0;
    for (int b = b0; b < b1; b++) s = __dadd_rn(s, __ldcg(partials + (size_t)b * KP + j));
    s_sl[q * KP + j] = s;
    __syncthreads();
    if (threadIdx.x < KP) {
        double t = 0.0;
        for (int i = 0; i < NS; i++) t = __dadd_rn(t, s_sl[i * KP + threadIdx.x]);
        totals[threadIdx.x] = t;
    }
    __syncthreads();
}

// Column-major (leading dimension ld) -> row-interleaved, padding zero.
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_pack(int n, int k, const double *__restrict__ src, long long ld,
                                                   double *__restrict__ dst)
{
    const long long total = (long long)n * KP;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT) {
        const long long i = e / KP;
        const int j = (int)(e % KP);
        dst[e] = j < k ? src[(long long)j * ld + i] : 0.0;
    }
}

// Row-interleaved -> column-major (the first k columns).
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_unpack(int n, int k, const double *__restrict__ src,
                                                     double *__restrict__ dst, long long ld)
{
    const long long total = (long long)n * KP;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT) {
        const long long i = e / KP;
        const int j = (int)(e % KP);
        if (j < k) dst[(long long)j * ld + i] = src[e];
    }
}

// x = 0, r = p = b (interleaved b given); per column ||b||^2 and the start
// state.
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_init(int n, int k, const double *__restrict__ bi, double *__restrict__ x,
                                                   double *__restrict__ r, double *__restrict__ p,
                                                   double *__restrict__ partials, MrState *st, double tol, int fixed,
                                                   int maxiter)
{
    __shared__ double sw[MR_NT / 32][MR_MAXK];
    __shared__ double tot[MR_MAXK];
    const long long total = (long long)n * KP;
    double b2 = 0.0;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT) {
        const double bv = bi[e];
        x[e] = 0.0;
        r[e] = bv;
        p[e] = bv;
        b2 = __dadd_rn(b2, __dmul_rn(bv, bv));
    }
    block_cols<KP>(b2, sw, partials + (size_t)blockIdx.x * KP);
    if (!mr_last_block(st)) return;
    sum_partials<KP>(partials, tot);
    if (threadIdx.x == 0) {
        int all = 1;
        for (int j = 0; j < KP; j++) {
            const double bb = tot[j], nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
            st->rho[j] = bb;
            st->nb[j] = nb;
            st->alpha[j] = 0.0;
            st->beta[j] = 0.0;
            st->iters[j] = 0;
            st->status[j] = MF_OK;
            const int d = j >= k || bb == 0.0 || (!fixed && sqrt(bb) <= tol * nb);
            st->done[j] = d;
            all &= d;
        }
        st->it = 0;
        st->stop = all || maxiter <= 0;
    }
}

// Y = A X over the row slots (X, Y row-interleaved with KP columns).  With
// PQ: skipped once the solve stopped; per-column partials of p.q (X = p,
// Y = q) and, in the last block, alpha per column.
template <int KP, bool PQ>
__global__ void __launch_bounds__(MR_NT, MR_SPMM_MINB) k_mr_spmm(MfTiles A, const int *__restrict__ sslot,
                                                   const uint16_t *__restrict__ smeta,
                                                   const double *__restrict__ sval, const double *__restrict__ X,
                                                   double *__restrict__ Y, double *__restrict__ partials, MrState *st)
{
    constexpr int QT = KP / 4;          // threads per row
    constexpr int RPB = MR_NT / QT;     // rows per block and pass
    __shared__ double sw[MR_NT / 32][MR_MAXK];
    __shared__ double tot[MR_MAXK];
    if (PQ && *(volatile int *)&st->stop) return;
    const int c0 = (threadIdx.x % QT) * 4;
    double pq[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * RPB + threadIdx.x / QT; i < A.rows; i += gridDim.x * RPB) {
        const int s = i >> 4, hl = i & 15;
        const int k0 = sslot[s], K = sslot[s + 1] - k0;
        const int *tcol = A.tile_columnidx + A.tile_ptr[s];
        double yd[4] = {0.0, 0.0, 0.0, 0.0}, part[4] = {0.0, 0.0, 0.0, 0.0};
        int prevj = -1;
#pragma unroll 4
        for (int kk = 0; kk < K; kk++) {
            const size_t e = (size_t)(k0 + kk) * MF_TILE + hl;
            const unsigned m = smeta[e];
            if (m == 0xFFFFu) continue;
            const double v = sval[e];
            const int tj = (int)(m >> 4);
            const long long col = (long long)tcol[tj] * MF_TILE + (m & 15u);
            const double2 xa = *(const double2 *)(X + col * KP + c0);
            const double2 xb = *(const double2 *)(X + col * KP + c0 + 2);
            if (tj != prevj) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    yd[q] = __dadd_rn(yd[q], part[q]);
                    part[q] = 0.0;
                }
                prevj = tj;
            }
            part[0] = __dadd_rn(part[0], __dmul_rn(xa.x, v));
            part[1] = __dadd_rn(part[1], __dmul_rn(xa.y, v));
            part[2] = __dadd_rn(part[2], __dmul_rn(xb.x, v));
            part[3] = __dadd_rn(part[3], __dmul_rn(xb.y, v));
        }
        double y[4];
#pragma unroll
        for (int q = 0; q < 4; q++) y[q] = __dadd_rn(yd[q], part[q]);
        double *yo = Y + (long long)i * KP + c0;
        *(double2 *)yo = make_double2(y[0], y[1]);
        *(double2 *)(yo + 2) = make_double2(y[2], y[3]);
        if (PQ) {
            const double *xo = X + (long long)i * KP + c0;
            const double2 pa = *(const double2 *)xo, pb = *(const double2 *)(xo + 2);
            pq[0] = __dadd_rn(pq[0], __dmul_rn(pa.x, y[0]));
            pq[1] = __dadd_rn(pq[1], __dmul_rn(pa.y, y[1]));
            pq[2] = __dadd_rn(pq[2], __dmul_rn(pb.x, y[2]));
            pq[3] = __dadd_rn(pq[3], __dmul_rn(pb.y, y[3]));
        }
    }
    if constexpr (PQ) {
        // lanes with the same column quad are QT apart
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int off = 16; off >= QT; off >>= 1) pq[q] = __dadd_rn(pq[q], __shfl_xor_sync(0xffffffffu, pq[q], off));
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane < QT)
#pragma unroll
            for (int q = 0; q < 4; q++) sw[w][c0 + q] = pq[q];
        __syncthreads();
        if (threadIdx.x < KP) {
            double t = 0.0;
            for (int i = 0; i < MR_NT / 32; i++) t = __dadd_rn(t, sw[i][threadIdx.x]);
            partials[(size_t)blockIdx.x * KP + threadIdx.x] = t;
        }
        if (!mr_last_block(st)) return;
        sum_partials<KP>(partials, tot);
        if (threadIdx.x < KP) {
            const int j = threadIdx.x;
            double al = 0.0;
            if (!st->done[j]) {
                const double d = tot[j];
                if (d != 0.0 && isfinite(d)) {
                    al = st->rho[j] / d;
                } else {
                    st->status[j] = MF_ERR_BREAKDOWN;
                    st->done[j] = 1;
                }
            }
            st->alpha[j] = al;
        }
    }
}

// x += alpha p, r -= alpha q; per-column r.r; the last block counts the
// iteration, tests convergence and sets beta and the stop flag.
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_update(int n, double *__restrict__ x, double *__restrict__ r,
                                                     const double *__restrict__ p, const double *__restrict__ q,
                                                     double *__restrict__ partials, MrState *st, double tol, int fixed,
                                                     int maxiter)
{
    __shared__ double sw[MR_NT / 32][MR_MAXK];
    __shared__ double tot[MR_MAXK];
    if (*(volatile int *)&st->stop) return;
    const double al = st->alpha[threadIdx.x % KP];
    const long long total = (long long)n * KP;
    double rr = 0.0;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT) {
        x[e] = fma(al, p[e], x[e]);
        const double ri = fma(-al, q[e], r[e]);
        r[e] = ri;
        rr = __dadd_rn(rr, __dmul_rn(ri, ri));
    }
    block_cols<KP>(rr, sw, partials + (size_t)blockIdx.x * KP);
    if (!mr_last_block(st)) return;
    sum_partials<KP>(partials, tot);
    if (threadIdx.x == 0) {
        int all = 1;
        for (int j = 0; j < KP; j++) {
            if (!st->done[j]) {
                const double rn = tot[j];
                st->iters[j]++;
                st->beta[j] = rn / st->rho[j];
                st->rho[j] = rn;
                if (rn == 0.0 || (!fixed && sqrt(rn) <= tol * st->nb[j])) {
                    st->done[j] = 1;
                    st->beta[j] = 0.0;
                }
            }
            all &= st->done[j];
        }
        st->it++;
        st->stop = all || st->it >= maxiter;
    }
}

// p = r + beta p (the same fused multiply-add as the single-vector CG).
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_pupdate(int n, const double *__restrict__ r, double *__restrict__ p,
                                                      const MrState *st)
{
    if (*(const volatile int *)&st->stop) return;
    const double bt = st->beta[threadIdx.x % KP];
    const long long total = (long long)n * KP;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT)
        p[e] = fma(bt, p[e], r[e]);
}

// ||b - A x|| per column (q = A x given); the last block stores them.
template <int KP>
__global__ void __launch_bounds__(MR_NT, MR_VEC_MINB) k_mr_resid(int n, const double *__restrict__ bi,
                                                    const double *__restrict__ q, double *__restrict__ partials,
                                                    MrState *st)
{
    __shared__ double sw[MR_NT / 32][MR_MAXK];
    __shared__ double tot[MR_MAXK];
    const long long total = (long long)n * KP;
    double d2 = 0.0;
    for (long long e = (long long)blockIdx.x * MR_NT + threadIdx.x; e < total; e += (long long)gridDim.x * MR_NT) {
        const double d = bi[e] - q[e];
        d2 = __dadd_rn(d2, __dmul_rn(d, d));
    }
    block_cols<KP>(d2, sw, partials + (size_t)blockIdx.x * KP);
    if (!mr_last_block(st)) return;
    sum_partials<KP>(partials, tot);
    if (threadIdx.x < KP) st->rtrue[threadIdx.x] = sqrt(tot[threadIdx.x]);
}

// Grid of a launch: the blocks the device holds at once (one wave; every
// block then takes an equal share of the grid-stride loop), at most MR_GRID
// (the partials buffer) and at most one block per MR_NT work items.  Fixed
// for a given kernel and device, so the partial sums are too.
template <class Kern>
int mr_grid(Kern kernel, long long work)
{
    int dev = 0, sms = 0, nb = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, MR_NT, 0) != cudaSuccess || nb < 1)
        nb = 1, sms = 148;
    const long long cap = std::min<long long>(MR_GRID, (long long)nb * sms);
    return (int)std::max(1ll, std::min<long long>(cap, (work + MR_NT - 1) / MR_NT));
}

template <int KP>
mf_status spmm_kp(mf_matrix m, const double *xi, double *yi, double *partials, MrState *st, bool pq, cudaStream_t s)
{
    const MfTiles &A = m->v;
    const int grid = mr_grid(k_mr_spmm<KP, true>, (long long)A.rows * (KP / 4));
    if (pq)
        k_mr_spmm<KP, true><<<grid, MR_NT, 0, s>>>(A, m->d_sslot, m->d_smeta, m->d_sval, xi, yi, partials, st);
    else
        k_mr_spmm<KP, false><<<grid, MR_NT, 0, s>>>(A, m->d_sslot, m->d_smeta, m->d_sval, xi, yi, partials, st);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

template <int KP>
mf_status spmm_cm(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, cudaStream_t s)
{
    const MfTiles &A = m->v;
    double *xi = nullptr, *yi = nullptr;
    const cudaError_t ea = pool_malloc_async(&xi, sizeof(double) * ((size_t)A.cols * KP + KP), s);
    const cudaError_t eb = pool_malloc_async(&yi, sizeof(double) * ((size_t)A.rows * KP + KP), s);
    if (ea != cudaSuccess || eb != cudaSuccess) {
        if (xi) cudaFreeAsync(xi, s);
        if (yi) cudaFreeAsync(yi, s);
        set_last_error("multi-vector SpMM: no device memory for %d columns", KP);
        return MF_ERR_NO_MEMORY;
    }
    mf_status st = MF_OK;
    k_mr_pack<KP><<<mr_grid(k_mr_pack<KP>, (long long)A.cols * KP), MR_NT, 0, s>>>(A.cols, k, X, ldx, xi);
    note_launch();
    if (cudaGetLastError() != cudaSuccess) st = MF_ERR_CUDA;
    if (st == MF_OK) st = spmm_kp<KP>(m, xi, yi, nullptr, nullptr, false, s);
    if (st == MF_OK) {
        k_mr_unpack<KP><<<mr_grid(k_mr_unpack<KP>, (long long)A.rows * KP), MR_NT, 0, s>>>(A.rows, k, yi, Y, ldy);
        note_launch();
        if (cudaGetLastError() != cudaSuccess) st = MF_ERR_CUDA;
    }
    cudaFreeAsync(xi, s);
    cudaFreeAsync(yi, s);
    if (st != MF_OK) set_last_error("multi-vector SpMM: kernel launch failed");
    return st;
}

template <int KP>
mf_status cg_multi_kp(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx, const mf_solve_opts &o,
                      mf_solve_report *reports, cudaStream_t s)
{
    const MfTiles &A = m->v;
    const int n = A.rows;
    const size_t E = (size_t)n * KP + KP;
    const int gv = mr_grid(k_mr_update<KP>, (long long)n * KP);
    const int gs = mr_grid(k_mr_spmm<KP, true>, (long long)n * (KP / 4));
    const int fixed = o.tol < 0.0;
    // workspace kept in the matrix handle: 5 interleaved vectors, the
    // partials, the state (each region 256-byte aligned)
    const size_t vec_bytes = (sizeof(double) * 5 * E + 255) / 256 * 256;
    const size_t part_bytes = (sizeof(double) * (size_t)MR_GRID * KP + 255) / 256 * 256;
    const size_t need = vec_bytes + part_bytes + sizeof(MrState);
    if (m->mr_work_bytes < need) {
        if (m->mr_work) cudaFree(m->mr_work);
        m->mr_work = nullptr;
        m->mr_work_bytes = 0;
        if (cudaMalloc(&m->mr_work, need) != cudaSuccess) {
            m->mr_work = nullptr;
            set_last_error("multi-RHS CG: no device memory for 5 x %zu vector entries", E);
            return MF_ERR_NO_MEMORY;
        }
        m->mr_work_bytes = need;
    }
    double *buf = (double *)m->mr_work;
    double *partials = (double *)((char *)m->mr_work + vec_bytes);
    MrState *st = (MrState *)((char *)m->mr_work + vec_bytes + part_bytes);
    double *bi = buf, *xi = buf + E, *ri = buf + 2 * E, *pi = buf + 3 * E, *qi = buf + 4 * E;
    auto launched = [&]() -> mf_status {
        note_launch();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            set_last_error("multi-RHS CG: %s", cudaGetErrorString(e));
            return MF_ERR_CUDA;
        }
        return MF_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    mf_status rc = MF_OK;
    MrState h;
    memset(&h, 0, sizeof(h));
    do {
        if (cudaMemsetAsync(st, 0, sizeof(MrState), s) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            set_last_error("multi-RHS CG: setup failed");
            rc = MF_ERR_CUDA;
            break;
        }
        cudaEventRecord(e0, s);
        k_mr_pack<KP><<<gv, MR_NT, 0, s>>>(n, k, B, ldb, bi);
        if ((rc = launched()) != MF_OK) break;
        k_mr_init<KP><<<gv, MR_NT, 0, s>>>(n, k, bi, xi, ri, pi, partials, st, o.tol, fixed, o.maxiter);
        if ((rc = launched()) != MF_OK) break;
        // batches of iterations; every launch returns at once after the stop
        int issued = 0, stop = 0;
        while (rc == MF_OK) {
            if (cudaMemcpyAsync(&stop, &st->stop, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                set_last_error("multi-RHS CG: %s", cudaGetErrorString(cudaGetLastError()));
                rc = MF_ERR_CUDA;
                break;
            }
            if (stop || issued >= o.maxiter) break;
            for (int t = 0; t < MR_BATCH && rc == MF_OK; t++) {
                k_mr_spmm<KP, true><<<gs, MR_NT, 0, s>>>(A, m->d_sslot, m->d_smeta, m->d_sval, pi, qi, partials, st);
                if ((rc = launched()) != MF_OK) break;
                k_mr_update<KP><<<gv, MR_NT, 0, s>>>(n, xi, ri, pi, qi, partials, st, o.tol, fixed, o.maxiter);
                if ((rc = launched()) != MF_OK) break;
                k_mr_pupdate<KP><<<gv, MR_NT, 0, s>>>(n, ri, pi, st);
                if ((rc = launched()) != MF_OK) break;
            }
            issued += MR_BATCH;
        }
        if (rc != MF_OK) break;
        // true residuals from the FP64 SpMM of x, then x to the caller
        if ((rc = spmm_kp<KP>(m, xi, qi, nullptr, nullptr, false, s)) != MF_OK) break;
        k_mr_resid<KP><<<gv, MR_NT, 0, s>>>(n, bi, qi, partials, st);
        if ((rc = launched()) != MF_OK) break;
        k_mr_unpack<KP><<<gv, MR_NT, 0, s>>>(n, k, xi, X, ldx);
        if ((rc = launched()) != MF_OK) break;
        cudaEventRecord(e1, s);
        if (cudaMemcpyAsync(&h, st, sizeof(MrState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            set_last_error("multi-RHS CG: %s", cudaGetErrorString(cudaGetLastError()));
            rc = MF_ERR_CUDA;
        }
    } while (false);
    float ms = 0.f;
    if (rc == MF_OK) cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc != MF_OK) return rc;
    // algorithmic bytes: per iteration the FP64 matrix stream once for all
    // columns and 11 vector streams of n x KP (SpMM: p in, q out; update: x,
    // p, q, r in, x, r out; p update: r, p in, p out)
    const long long T = A.tilenum;
    const long long per_it = (long long)A.nnz * 9 + 24 * T + 16LL * n + 88LL * n * KP;
    mf_status ret = MF_OK;
    for (int j = 0; j < k; j++) {
        mf_solve_report &r = reports[j];
        memset(&r, 0, sizeof(r));
        r.iterations = h.iters[j];
        r.relres = sqrt(h.rho[j]) / h.nb[j];
        r.relres_true = h.rtrue[j] / h.nb[j];
        r.kernel_ms = ms;
        r.bytes_moved = per_it * h.it;
        r.grid_ctas = gs;
        r.layout = 1;
        int stc = h.status[j];
        if (stc == MF_OK && !fixed && !h.done[j]) stc = MF_ERR_NOT_CONVERGED;
        r.status = stc;
        if (stc != MF_OK && ret == MF_OK) ret = (mf_status)stc;
    }
    if (ret == MF_ERR_NOT_CONVERGED) set_last_error("multi-RHS CG: maxiter reached before the tolerance");
    if (ret == MF_ERR_BREAKDOWN) set_last_error("multi-RHS CG breakdown");
    return ret;
}

int kp_for(int k) { return k <= 4 ? 4 : k <= 8 ? 8 : 16; }

}  // namespace

mf_status spmm_multi(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, cudaStream_t s)
{
    MF_TRY(build_slots(m, s));
    if (m->slots_state != 1) {
        set_last_error("multi-vector SpMM: the matrix has no row-slot layout");
        return MF_ERR_UNSUPPORTED;
    }
    switch (kp_for(k)) {
    case 4: return spmm_cm<4>(m, k, X, ldx, Y, ldy, s);
    case 8: return spmm_cm<8>(m, k, X, ldx, Y, ldy, s);
    default: return spmm_cm<16>(m, k, X, ldx, Y, ldy, s);
    }
}

mf_status cg_multi(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx, const mf_solve_opts &o,
                   mf_solve_report *reports, cudaStream_t s)
{
    MF_TRY(build_slots(m, s));
    if (m->slots_state != 1) {
        set_last_error("multi-RHS CG: the matrix has no row-slot layout");
        return MF_ERR_UNSUPPORTED;
    }
    switch (kp_for(k)) {
    case 4: return cg_multi_kp<4>(m, k, B, ldb, X, ldx, o, reports, s);
    case 8: return cg_multi_kp<8>(m, k, B, ldb, X, ldx, o, reports, s);
    default: return cg_multi_kp<16>(m, k, B, ldb, X, ldx, o, reports, s);
    }
}

}  // namespace mf
