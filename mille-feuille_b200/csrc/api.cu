// api.cu -- the C ABI (include/mf.h): handles, status codes, host/device
// entry points.  No call aborts; every CUDA error becomes an mf_status.
#include <atomic>
#include <mutex>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>

#include "mf_internal.h"

namespace mf {

static thread_local char g_err[1024] = "";
static std::atomic<long long> g_launches{0};

void note_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

cudaError_t pool_malloc_async(void **p, size_t bytes, cudaStream_t s)
{
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, s);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props;
            memset(&props, 0, sizeof(props));
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&pools[dev], &props);
            if (e != cudaSuccess) {
                pools[dev] = nullptr;
                return e;
            }
            uint64_t keep = 256ull << 20;  // up to 256 MiB stays in the pool across synchronisations
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

void set_last_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

mf_status ensure_work(mf_matrix m, size_t bytes)
{
    if (m->work_bytes >= bytes) return MF_OK;
    if (m->work) cudaFree(m->work);
    m->work = nullptr;
    m->work_bytes = 0;
    MF_CUDA(cudaMalloc(&m->work, bytes));
    m->work_bytes = bytes;
    return MF_OK;
}

mf_status cg_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                   double *history, cudaStream_t s);
mf_status bicgstab_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep,
                         double *history, cudaStream_t s);
mf_status spmm_multi(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, cudaStream_t s);
mf_status cg_multi(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx, const mf_solve_opts &o,
                   mf_solve_report *reports, cudaStream_t s);

static mf_status check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_last_error("no CUDA device: %s", cudaGetErrorString(e));
        return MF_ERR_NO_DEVICE;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
        set_last_error("libmf is built for sm_100a (B200); device has compute capability %d.x", major);
        return MF_ERR_NO_DEVICE;
    }
    return MF_OK;
}

}  // namespace mf

using namespace mf;

extern "C" {

const char *mf_last_error(void) { return g_err; }
const char *mf_version(void) { return "mille-feuille-b200 0.1 (sm_100a)"; }
long long mf_kernel_launches(void) { return g_launches.load(); }

void mf_free_host(void *p) { free(p); }

mf_status mf_matrix_create(int rowA, int colA, const int *rowptr, const int *colidx, const double *val,
                           const float *val_low, int on_device, void *stream, mf_matrix *out)
{
    g_err[0] = 0;
    if (!out || !rowptr || rowA < 0 || colA < 0 || (rowA > 0 && (!colidx || !val))) {
        set_last_error("mf_matrix_create: invalid arguments");
        return MF_ERR_INVALID_ARG;
    }
    *out = nullptr;
    MF_TRY(check_device());
    cudaStream_t s = (cudaStream_t)stream;
    const int *d_rp = rowptr, *d_ci = colidx;
    const double *d_v = val;
    const float *d_vl = val_low;
    void *tmp = nullptr;
    if (!on_device) {
        const int rp0 = rowptr[0];
        const long long nnz_end = rowptr[rowA];
        if (nnz_end < rp0) {
            set_last_error("rowptr[rowA] < rowptr[0]");
            return MF_ERR_INVALID_ARG;
        }
        size_t b_rp = sizeof(int) * (rowA + 1), b_ci = sizeof(int) * nnz_end, b_v = sizeof(double) * nnz_end,
               b_vl = val_low ? sizeof(float) * nnz_end : 0;
        MF_CUDA(cudaMalloc(&tmp, b_rp + b_ci + b_v + b_vl + 64));
        char *c = (char *)tmp;
        double *dv = (double *)c;
        int *dci = (int *)(c + b_v);
        int *drp = (int *)(c + b_v + b_ci);
        float *dvl = val_low ? (float *)(c + b_v + b_ci + b_rp + ((4 - (b_rp & 3)) & 3)) : nullptr;
        cudaError_t e = cudaMemcpyAsync(drp, rowptr, b_rp, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nnz_end > 0) e = cudaMemcpyAsync(dci, colidx, b_ci, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nnz_end > 0) e = cudaMemcpyAsync(dv, val, b_v, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && val_low && nnz_end > 0) e = cudaMemcpyAsync(dvl, val_low, b_vl, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            cudaFree(tmp);
            set_last_error("H2D copy: %s", cudaGetErrorString(e));
            return MF_ERR_CUDA;
        }
        d_rp = drp;
        d_ci = dci;
        d_v = dv;
        d_vl = dvl;
    }
    mf_matrix m = new mf_matrix_s();
    memset(&m->v, 0, sizeof(m->v));
    cudaGetDevice(&m->device);
    mf_status st = build_tiles(m, rowA, colA, d_rp, d_ci, d_v, d_vl, s);
    if (tmp) {
        cudaStreamSynchronize(s);
        cudaFree(tmp);
    }
    if (st != MF_OK) {
        mf_matrix_destroy(m);
        return st;
    }
    *out = m;
    return MF_OK;
}

mf_status mf_matrix_destroy(mf_matrix m)
{
    if (!m) return MF_OK;
    void *bufs[] = {m->d_tile_ptr, m->d_tile_columnidx, m->d_tile_nnz, m->d_csrptr_offset, m->d_blknnznnz, m->d_val,
                    m->d_val_low, m->d_col, m->d_ptr, m->d_cidx, m->d_f16, m->d_i8, m->d_class, m->d_f16ok,
                    m->d_nonzero_row_new, m->d_tile_rowidx, m->d_block_signal, m->d_blockrowid_new, m->d_blockcsr_ptr_new, m->d_rbb_rowidx,
                    m->d_rbb_colstart, m->d_rbb_colstop, m->d_part, m->d_cta_chunk, m->d_chunks, m->work, m->host_io,
                    m->d_wcls, m->d_poff, m->d_pay, m->d_resid, m->d_pol, m->d_sslot, m->d_smeta, m->d_sval,
                    m->d_shdr, m->d_spay, m->d_scta_chunk, m->d_schunks, m->d_spos, m->d_sdesc, m->mr_work,
                    m->mr_io, m->d_tc_index, m->d_tc_dense};
    for (void *p : bufs)
        if (p) cudaFree(p);
    delete m;
    return MF_OK;
}

mf_status mf_matrix_get_info(mf_matrix m, mf_matrix_info *info)
{
    if (!m || !info) return MF_ERR_INVALID_ARG;
    memset(info, 0, sizeof(*info));
    info->rows = m->v.rows;
    info->cols = m->v.cols;
    info->nnz = m->v.nnz;
    info->tilem = m->v.tilem;
    info->tilen = m->v.tilen;
    info->tilenum = m->v.tilenum;
    info->csrsize = m->v.nnz;
    info->csrptrlen = m->v.csrptrlen;
    info->nonzero_rows = m->nonzero_rows;
    info->rowblkblock = m->rowblkblock;
    for (int c = 0; c < 5; c++) info->class_tiles[c] = m->class_tiles[c];
    info->max_tile_nnz = m->max_tile_nnz;
    info->device_bytes = m->device_bytes;
    return MF_OK;
}

static bool array_desc(mf_matrix m, const char *name, const void **ptr, size_t *bytes)
{
    const size_t T = m->v.tilenum, nnz = m->v.nnz, tilem = m->v.tilem;
    struct D {
        const char *n;
        const void *p;
        size_t b;
    } tab[] = {
        {"tile_ptr", m->d_tile_ptr, 4 * (tilem + 1)},
        {"tile_columnidx", m->d_tile_columnidx, 4 * T},
        {"tile_nnz", m->d_tile_nnz, 4 * (T + 1)},
        {"blknnz", m->d_tile_nnz, 4 * (T + 1)},
        {"csr_offset", m->d_tile_nnz, 4 * (T + 1)},
        {"ptroffset1", m->d_tile_nnz, 4 * T},
        {"csrptr_offset", m->d_csrptr_offset, 4 * (T + 1)},
        {"ptroffset2", m->d_csrptr_offset, 4 * T},
        {"blknnznnz", m->d_blknnznnz, T + 1},
        {"Blockcsr_Val", m->d_val, 8 * nnz},
        {"Blockcsr_Val_Low", m->d_val_low, 4 * nnz},
        {"Tile_csr_Col", m->d_col, nnz},
        {"Blockcsr_Ptr", m->d_ptr, (size_t)m->v.csrptrlen},
        {"csr_compressedIdx", m->d_cidx, (nnz + 1) / 2},
        {"nonzero_row_new", m->d_nonzero_row_new, 4 * (T + 1)},
        {"tile_rowidx", m->d_tile_rowidx, 4 * T},
        {"block_signal", m->d_block_signal, 4 * (tilem + 1)},
        {"blockrowid_new", m->d_blockrowid_new, (size_t)m->nonzero_rows + 1},
        {"blockcsr_ptr_new", m->d_blockcsr_ptr_new, (size_t)m->nonzero_rows + 1},
        {"rowblkblock_rowidx", m->d_rbb_rowidx, 4 * (size_t)m->rowblkblock},
        {"rowblkblock_colstart", m->d_rbb_colstart, 4 * (size_t)m->rowblkblock},
        {"rowblkblock_colstop", m->d_rbb_colstop, 4 * (size_t)m->rowblkblock},
        {"tile_class", m->d_class, T},
        {"tile_f16ok", m->d_f16ok, T},
        {"payload_f16", m->d_f16, 2 * nnz},
        {"payload_i8", m->d_i8, nnz},
    };
    for (auto &d : tab)
        if (!strcmp(d.n, name)) {
            *ptr = d.p;
            *bytes = d.b;
            return true;
        }
    return false;
}

mf_status mf_matrix_array_bytes(mf_matrix m, const char *name, size_t *bytes)
{
    const void *p;
    if (!m || !name || !bytes || !array_desc(m, name, &p, bytes)) {
        set_last_error("unknown array name");
        return MF_ERR_INVALID_ARG;
    }
    return MF_OK;
}

mf_status mf_matrix_export(mf_matrix m, const char *name, void *host_dst, size_t bytes)
{
    const void *p;
    size_t b;
    if (!m || !name || !array_desc(m, name, &p, &b)) {
        set_last_error("unknown array name");
        return MF_ERR_INVALID_ARG;
    }
    if (bytes != b || (b > 0 && !host_dst)) {
        set_last_error("export %s: expected %zu bytes, got %zu", name, b, bytes);
        return MF_ERR_INVALID_ARG;
    }
    if (b == 0) return MF_OK;
    MF_CUDA(cudaMemcpy(host_dst, p, b, cudaMemcpyDeviceToHost));
    return MF_OK;
}

static __global__ void k_encode(int n, const unsigned char *__restrict__ col, unsigned char *__restrict__ out)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < (n + 1) / 2; p += gridDim.x * blockDim.x) {
        unsigned char hi = col[2 * p];
        unsigned char lo = (2 * p + 1 < n) ? col[2 * p + 1] : 0;
        out[p] = (unsigned char)((hi << 4) + lo);
    }
}

mf_status mf_encode_column_index(mf_matrix m, void *stream)
{
    if (!m) return MF_ERR_INVALID_ARG;
    const int n = m->v.nnz;
    if (n == 0) return MF_OK;
    int grid = ceil_div((n + 1) / 2, 256);
    if (grid > 148 * 16) grid = 148 * 16;
    k_encode<<<grid, 256, 0, (cudaStream_t)stream>>>(n, m->d_col, m->d_cidx);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

mf_status mf_spmv(mf_matrix m, const double *x, double *y, void *stream)
{
    if (!m || (m->v.rows > 0 && (!x || !y))) return MF_ERR_INVALID_ARG;
    return spmv_fp64(m->v, x, y, (cudaStream_t)stream);
}

void mf_solve_opts_default(mf_solve_opts *o)
{
    if (!o) return;
    o->maxiter = 20000;
    o->tol = 1e-10;
    o->policy = MF_POLICY_FP64;
    o->refine_delta = 0.1;
    o->wait_budget_s = 5.0;
    o->record_history = 0;
    o->phase_times = 0;
    o->precond = 0;
}

static mf_status solve_common(bool bicg, mf_matrix m, const double *b, double *x, const mf_solve_opts *opts,
                              mf_solve_report *report, double *history, void *stream)
{
    g_err[0] = 0;
    if (!m || !b || !x) {
        set_last_error("solve: null argument");
        return MF_ERR_INVALID_ARG;
    }
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    if (opts) o = *opts;
    if (o.maxiter < 0 || o.wait_budget_s <= 0 || o.policy < 0 || o.policy > MF_POLICY_STATIC_FP16 || o.precond < 0 ||
        o.precond > 1) {
        set_last_error("solve: maxiter < 0, wait budget <= 0, unknown policy or unknown preconditioner");
        return MF_ERR_INVALID_ARG;
    }
    if (bicg && o.precond) {
        set_last_error("solve: the Jacobi preconditioner is available for CG only");
        return MF_ERR_UNSUPPORTED;
    }
    if (m->v.rows != m->v.cols) {
        set_last_error("solve: matrix is %d x %d, a square system is required", m->v.rows, m->v.cols);
        return MF_ERR_INVALID_ARG;
    }
    mf_solve_report rep;
    memset(&rep, 0, sizeof(rep));
    mf_status st;
    if (m->v.rows == 0) {
        st = MF_OK;
    } else if (!bicg && o.policy == MF_POLICY_LEARNED && !m->policy_loaded) {
        set_last_error("learned policy requested but no policy is loaded (mf_policy_load / mf_policy_train)");
        st = MF_ERR_UNSUPPORTED;
    } else {
        st = bicg ? bicgstab_solve(m, b, x, o, rep, history, (cudaStream_t)stream)
                  : cg_solve(m, b, x, o, rep, history, (cudaStream_t)stream);
    }
    rep.status = st;
    if (report) *report = rep;
    return st;
}

static mf_status solve_host_common(bool bicg, mf_matrix m, const double *b_host, double *x_host,
                                   const mf_solve_opts *opts, mf_solve_report *report)
{
    if (!m || !b_host || !x_host) return MF_ERR_INVALID_ARG;
    const size_t n = m->v.rows;
    if (m->host_io_n < n) {
        if (m->host_io) cudaFree(m->host_io);
        m->host_io = nullptr;
        m->host_io_n = 0;
        MF_CUDA(cudaMalloc(&m->host_io, sizeof(double) * (2 * n + 2)));
        m->host_io_n = n;
    }
    double *db = m->host_io, *dx = m->host_io + n + 1;
    cudaStream_t s = 0;
    cudaError_t e = cudaMemcpyAsync(db, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        set_last_error("H2D: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    mf_status st = solve_common(bicg, m, db, dx, opts, report, nullptr, s);
    e = cudaMemcpyAsync(x_host, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_last_error("D2H: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    return st;
}

mf_status mf_cg_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts *opts, mf_solve_report *report,
                      double *history, void *stream)
{
    return solve_common(false, m, b, x, opts, report, history, stream);
}

mf_status mf_cg_solve_host(mf_matrix m, const double *b_host, double *x_host, const mf_solve_opts *opts,
                           mf_solve_report *report)
{
    return solve_host_common(false, m, b_host, x_host, opts, report);
}

mf_status mf_bicgstab_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts *opts,
                            mf_solve_report *report, double *history, void *stream)
{
    return solve_common(true, m, b, x, opts, report, history, stream);
}

mf_status mf_bicgstab_solve_host(mf_matrix m, const double *b_host, double *x_host, const mf_solve_opts *opts,
                                 mf_solve_report *report)
{
    return solve_host_common(true, m, b_host, x_host, opts, report);
}

mf_status mf_spmm(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, void *stream)
{
    g_err[0] = 0;
    if (!m || k < 1 || k > 16) {
        set_last_error("spmm: null matrix or k = %d outside 1..16", k);
        return MF_ERR_INVALID_ARG;
    }
    if (ldx < m->v.cols || ldy < m->v.rows || (m->v.rows > 0 && (!X || !Y))) {
        set_last_error("spmm: null array or leading dimension shorter than the matrix");
        return MF_ERR_INVALID_ARG;
    }
    if (m->v.rows == 0) return MF_OK;
    return spmm_multi(m, k, X, ldx, Y, ldy, (cudaStream_t)stream);
}

mf_status mf_cg_solve_multi(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx,
                            const mf_solve_opts *opts, mf_solve_report *reports, void *stream)
{
    g_err[0] = 0;
    if (!m || k < 1 || k > 16 || !reports) {
        set_last_error("multi-RHS solve: null matrix or reports, or k = %d outside 1..16", k);
        return MF_ERR_INVALID_ARG;
    }
    mf_solve_opts o;
    mf_solve_opts_default(&o);
    if (opts) o = *opts;
    if (o.maxiter < 0 || o.policy < 0 || o.policy > MF_POLICY_STATIC_FP16 || o.precond < 0 || o.precond > 1) {
        set_last_error("multi-RHS solve: maxiter < 0, unknown policy or unknown preconditioner");
        return MF_ERR_INVALID_ARG;
    }
    if (o.policy != MF_POLICY_FP64 || o.precond) {
        set_last_error("multi-RHS solve: FP64 policy without preconditioner only");
        return MF_ERR_UNSUPPORTED;
    }
    if (m->v.rows != m->v.cols) {
        set_last_error("multi-RHS solve: matrix is %d x %d, a square system is required", m->v.rows, m->v.cols);
        return MF_ERR_INVALID_ARG;
    }
    if (ldb < m->v.rows || ldx < m->v.rows || (m->v.rows > 0 && (!B || !X))) {
        set_last_error("multi-RHS solve: null array or leading dimension shorter than the matrix");
        return MF_ERR_INVALID_ARG;
    }
    for (int j = 0; j < k; j++) memset(&reports[j], 0, sizeof(mf_solve_report));
    if (m->v.rows == 0) return MF_OK;
    return cg_multi(m, k, B, ldb, X, ldx, o, reports, (cudaStream_t)stream);
}

mf_status mf_cg_solve_multi_host(mf_matrix m, int k, const double *B_host, double *X_host,
                                 const mf_solve_opts *opts, mf_solve_report *reports)
{
    g_err[0] = 0;
    if (!m || !B_host || !X_host || k < 1 || k > 16) {
        set_last_error("multi-RHS solve: null argument or k = %d outside 1..16", k);
        return MF_ERR_INVALID_ARG;
    }
    const size_t n = m->v.rows, bytes = sizeof(double) * n * (size_t)k;
    if (n == 0) return mf_cg_solve_multi(m, k, nullptr, 0, nullptr, 0, opts, reports, nullptr);
    cudaStream_t s = 0;
    if (m->mr_io_bytes < 2 * bytes) {
        if (m->mr_io) cudaFree(m->mr_io);
        m->mr_io = nullptr;
        m->mr_io_bytes = 0;
        MF_CUDA(cudaMalloc(&m->mr_io, 2 * bytes));
        m->mr_io_bytes = 2 * bytes;
    }
    double *dB = (double *)m->mr_io, *dX = dB + n * (size_t)k;
    cudaError_t e = cudaMemcpyAsync(dB, B_host, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        set_last_error("H2D: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    const mf_status st = mf_cg_solve_multi(m, k, dB, (int)n, dX, (int)n, opts, reports, s);
    // X is only written when the solve ran: a call rejected before its
    // kernels (bad options, an unsupported policy) leaves X_host untouched.
    if (st != MF_OK && st != MF_ERR_NOT_CONVERGED && st != MF_ERR_BREAKDOWN) {
        cudaStreamSynchronize(s);
        return st;
    }
    e = cudaMemcpyAsync(X_host, dX, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_last_error("D2H: %s", cudaGetErrorString(e));
        return MF_ERR_CUDA;
    }
    return st;
}

}  // extern "C"
