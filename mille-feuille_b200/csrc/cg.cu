// cg.cu -- single persistent CG kernel (FP64 policy).
//
// The reference runs CG inside one persistent kernel whose warps sync through
// atomic counters and spin-waits, with atomicAdd(double) dot products
// (src/Mille-feuille-cg.h:168-350, 352-580, 1109-1343).  Here:
//   * one cooperative launch, grid = resident CTAs (never more), so every
//     grid-wide wait can finish; every wait is bounded in time and reports
//     MF_ERR_TIMEOUT through a status word instead of hanging;
//   * each CTA owns a contiguous, cost-balanced range of 16-row strips for the
//     SpMV and for the vector updates, so only p crosses CTAs;
//   * dot products are deterministic: per-thread sequential sums, a fixed
//     CTA tree, per-CTA partials in fixed slots, and every CTA sums the
//     partials in the same order -- no double atomics, repeatable runs;
//   * the loop stops on ||r|| <= tol ||b|| (tol < 0: fixed iteration count,
//     the reference's behaviour).
#include <cooperative_groups.h>

#include "spmv_core.cuh"

namespace mf {
namespace {

constexpr int CG_NT = 256;

struct CgArgs {
    MfTiles A;
    const int *part;
    const double *b;
    double *x, *r, *p, *q;
    double *partials;  // [3][G]
    unsigned long long *bar;
    int *status;
    double *hist;      // optional [maxiter+1]
    double *out;       // [0] rho, [1] bb, [2] iterations
    int maxiter;
    double tol;
    int fixed;
    unsigned long long budget_ns;
};

struct GridCtx {
    unsigned long long epoch;
    bool ok;
};

template <int NT>
__device__ __forceinline__ double grid_sum(const CgArgs &a, double local, int slot, GridCtx &gc, double *s_warp)
{
    const int G = gridDim.x;
    double cta = block_sum<NT>(local, s_warp);
    if (threadIdx.x == 0) a.partials[slot * G + blockIdx.x] = cta;
    gc.epoch++;
    gc.ok = gc.ok && grid_barrier(a.bar, gc.epoch * (unsigned long long)G, a.status, a.budget_ns);
    __shared__ double s_res;
    if (threadIdx.x < 32) {
        double s = warp_sum_partials(a.partials + slot * G, G);
        if (threadIdx.x == 0) s_res = s;
    }
    __syncthreads();
    return s_res;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_cg_fp64(CgArgs a)
{
    __shared__ double s_warp[NT / 32];
    const MfTiles &A = a.A;
    const int sb = a.part[blockIdx.x], se = a.part[blockIdx.x + 1];
    const int r16 = threadIdx.x & 15;
    const int sstep = NT / MF_TILE;
    GridCtx gc{0ull, true};

    double loc = 0.0;
    for (int bi = sb + (threadIdx.x >> 4); bi < se; bi += sstep) {
        const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
        if (r16 < rowlen) {
            const int i = bi * MF_TILE + r16;
            const double bv = a.b[i];
            a.x[i] = 0.0;
            a.r[i] = bv;
            a.p[i] = bv;
            loc = __dadd_rn(loc, __dmul_rn(bv, bv));
        }
    }
    const double bb = grid_sum<NT>(a, loc, 0, gc, s_warp);
    const double nb = sqrt(bb) > 0.0 ? sqrt(bb) : 1.0;
    double rho = bb;
    int it = 0;
    if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[0] = sqrt(rho) / nb;
    while (gc.ok && it < a.maxiter) {
        if (!a.fixed && sqrt(rho) <= a.tol * nb) break;
        // q = A p over own strips, p.q partial
        loc = 0.0;
        for (int bi = sb + (threadIdx.x >> 4); bi < se; bi += sstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (r16 < rowlen) {
                const int i = bi * MF_TILE + r16;
                const double qi = row_fp64(A, bi, r16, rowlen, a.p);
                a.q[i] = qi;
                loc = __dadd_rn(loc, __dmul_rn(a.p[i], qi));
            }
        }
        const double pq = grid_sum<NT>(a, loc, 1, gc, s_warp);
        if (!gc.ok) break;
        if (!(pq != 0.0) || !isfinite(pq)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(a.status, DEV_OK, DEV_BREAKDOWN);
            break;
        }
        const double alpha = rho / pq;
        loc = 0.0;
        for (int bi = sb + (threadIdx.x >> 4); bi < se; bi += sstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (r16 < rowlen) {
                const int i = bi * MF_TILE + r16;
                a.x[i] = fma(alpha, a.p[i], a.x[i]);
                const double ri = fma(-alpha, a.q[i], a.r[i]);
                a.r[i] = ri;
                loc = __dadd_rn(loc, __dmul_rn(ri, ri));
            }
        }
        const double rho_new = grid_sum<NT>(a, loc, 2, gc, s_warp);
        if (!gc.ok) break;
        const double beta = rho_new / rho;
        rho = rho_new;
        for (int bi = sb + (threadIdx.x >> 4); bi < se; bi += sstep) {
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            if (r16 < rowlen) {
                const int i = bi * MF_TILE + r16;
                a.p[i] = fma(beta, a.p[i], a.r[i]);
            }
        }
        gc.epoch++;
        gc.ok = grid_barrier(a.bar, gc.epoch * (unsigned long long)gridDim.x, a.status, a.budget_ns);
        it++;
        if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[it] = sqrt(rho) / nb;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = rho;
        a.out[1] = bb;
        a.out[2] = (double)it;
    }
}

// ||b - A x||^2 and ||b||^2 from y = A x, deterministic (per-CTA partials,
// summed in order by one CTA).
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
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int i = 0; i < nblk; i++) {
            a += part[2 * i];
            b += part[2 * i + 1];
        }
        out[0] = a;
        out[1] = b;
    }
}

}  // namespace

// Workspace layout for one solve (cached on the matrix handle).
struct CgWork {
    double *r, *p, *q, *partials, *out, *ax, *rpart;
    unsigned long long *bar;
    int *status;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

mf_status cg_resources(mf_matrix m, int G, CgWork &w)
{
    const size_t n = (size_t)m->v.tilem * MF_TILE + 16;
    size_t off = 0;
    size_t o_r = off; off += align256(n * 8);
    size_t o_p = off; off += align256(n * 8);
    size_t o_q = off; off += align256(n * 8);
    size_t o_ax = off; off += align256(n * 8);
    size_t o_part = off; off += align256((size_t)3 * G * 8);
    size_t o_rp = off; off += align256((size_t)2 * 1024 * 8);
    size_t o_out = off; off += align256(8 * 8);
    size_t o_bar = off; off += align256(8);
    size_t o_st = off; off += align256(8);
    MF_TRY(ensure_work(m, off));
    char *base = (char *)m->work;
    w.r = (double *)(base + o_r);
    w.p = (double *)(base + o_p);
    w.q = (double *)(base + o_q);
    w.ax = (double *)(base + o_ax);
    w.partials = (double *)(base + o_part);
    w.rpart = (double *)(base + o_rp);
    w.out = (double *)(base + o_out);
    w.bar = (unsigned long long *)(base + o_bar);
    w.status = (int *)(base + o_st);
    return MF_OK;
}

int cg_grid(mf_matrix m)
{
    static int max_ctas = -1;
    if (max_ctas < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg_fp64<CG_NT>, CG_NT, 0);
        max_ctas = sms * (per > 0 ? per : 1);
    }
    int want = ceil_div(m->v.tilem, CG_NT / MF_TILE);
    if (want < 1) want = 1;
    return want < max_ctas ? want : max_ctas;
}

mf_status true_residual(mf_matrix m, const double *b, const double *x, CgWork &w, double *relres, cudaStream_t s)
{
    const int n = m->v.rows;
    MF_TRY(spmv_fp64(m->v, x, w.ax, s));
    const int nblk = 512;
    k_resid_partials<<<nblk, 256, 0, s>>>(n, b, w.ax, w.rpart);
    note_launch();
    MF_CUDA(cudaGetLastError());
    k_resid_final<<<1, 32, 0, s>>>(nblk, w.rpart, w.out + 4);
    note_launch();
    MF_CUDA(cudaGetLastError());
    double h[2];
    MF_CUDA(cudaMemcpyAsync(h, w.out + 4, sizeof(h), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    *relres = h[1] > 0 ? sqrt(h[0]) / sqrt(h[1]) : sqrt(h[0]);
    return MF_OK;
}

mf_status cg_solve_fp64(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                        double *history, cudaStream_t s)
{
    const int G = cg_grid(m);
    MF_TRY(strip_partition(m, G, s));
    CgWork w;
    MF_TRY(cg_resources(m, G, w));
    MF_CUDA(cudaMemsetAsync(w.bar, 0, sizeof(unsigned long long), s));
    MF_CUDA(cudaMemsetAsync(w.status, 0, sizeof(int), s));
    CgArgs a;
    a.A = m->v;
    a.part = m->d_part;
    a.b = b;
    a.x = x;
    a.r = w.r;
    a.p = w.p;
    a.q = w.q;
    a.partials = w.partials;
    a.bar = w.bar;
    a.status = w.status;
    a.hist = (o.record_history && history) ? history : nullptr;
    a.out = w.out;
    a.maxiter = o.maxiter;
    a.tol = o.tol;
    a.fixed = o.tol < 0 ? 1 : 0;
    a.budget_ns = (unsigned long long)(o.wait_budget_s * 1e9);
    cudaEvent_t e0, e1;
    MF_CUDA(cudaEventCreate(&e0));
    MF_CUDA(cudaEventCreate(&e1));
    MF_CUDA(cudaEventRecord(e0, s));
    void *args[] = {&a};
    note_launch();
    MF_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg_fp64<CG_NT>, dim3(G), dim3(CG_NT), args, 0, s));
    MF_CUDA(cudaEventRecord(e1, s));
    double h_out[3];
    int h_status = 0;
    MF_CUDA(cudaMemcpyAsync(h_out, w.out, sizeof(h_out), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaMemcpyAsync(&h_status, w.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rep.iterations = (int)h_out[2];
    rep.grid_ctas = G;
    rep.kernel_ms = ms;
    const double nb = h_out[1] > 0 ? sqrt(h_out[1]) : 1.0;
    rep.relres = sqrt(h_out[0]) / nb;
    rep.refinements = 0;
    const long long n = m->v.rows, T = m->v.tilenum, nnz = m->v.nnz;
    rep.bytes_moved = (long long)rep.iterations * (nnz * 9 + 24 * T + 16 * n + 72 * n);
    MF_TRY(true_residual(m, b, x, w, &rep.relres_true, s));
    if (h_status != 0) {
        rep.status = h_status;
        set_last_error(h_status == MF_ERR_TIMEOUT ? "grid-wide wait exceeded its budget" : "CG breakdown");
        return (mf_status)h_status;
    }
    if (!a.fixed && !(rep.relres <= o.tol)) {
        rep.status = MF_ERR_NOT_CONVERGED;
        return MF_ERR_NOT_CONVERGED;
    }
    rep.status = MF_OK;
    return MF_OK;
}

}  // namespace mf
