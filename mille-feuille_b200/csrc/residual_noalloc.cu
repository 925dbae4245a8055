// residual_noalloc.cu -- mf_residual_norm without any device allocation.
//
// Some callers may not allocate device memory on the path that checks a
// solve: services that size all device memory once at start-up, callers
// whose device memory must come from their own allocator, and callers that
// cannot accept the device-wide synchronisation cudaMalloc/cudaFree may
// cause while other streams are running.  For them this entry point keeps
// the per-strip partials of the residual check in a fixed array that lives
// in the library's own device image, so the call allocates nothing.
//
// The array holds the partials of at most MF_NOALLOC_MAX_STRIPS 16-row
// strips (1 MiB, present on every GPU that loads the library until the
// process exits); larger matrices are rejected with MF_ERR_INVALID_ARG.
// Every call on a device uses the same array: calls whose kernels overlap on
// the GPU (different streams) race on it and must be ordered by the caller.
// Each call writes every partial it reads before reading it, so no clearing
// is needed between calls.
#include <mutex>

#include "mf_internal.h"

#define MF_NOALLOC_MAX_STRIPS 65536

namespace {

// File-scope scratch: two doubles (squared residual, squared rhs) per strip.
static __device__ __align__(256) double g_noalloc_part[2 * MF_NOALLOC_MAX_STRIPS];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
double *g_part_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (set up once per
// device, with that device current).  In host code the array's name is only
// a host-side stand-in, so its device address must come from the runtime.
// The matrix must live on the current device: its pointers are used by
// kernels launched there.
mf_status scratch_address(int matrix_device, double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        mf::set_last_error("mf_residual_norm_noalloc: no usable current device (%s)", cudaGetErrorString(e));
        return MF_ERR_NO_DEVICE;
    }
    if (dev != matrix_device) {
        mf::set_last_error("mf_residual_norm_noalloc: the matrix lives on device %d but device %d is current",
                           matrix_device, dev);
        return MF_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_part_ptr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_part);
        if (e != cudaSuccess || !p) {
            mf::set_last_error("mf_residual_norm_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return MF_ERR_CUDA;
        }
        g_part_ptr[dev] = p;
    }
    *out = g_part_ptr[dev];
    return MF_OK;
}

}  // namespace

extern "C" mf_status mf_residual_norm_noalloc(mf_matrix m, const double *b, const double *x, double *out,
                                              void *stream)
{
    if (!m || !b || !x || !out) {
        mf::set_last_error("mf_residual_norm_noalloc: null argument");
        return MF_ERR_INVALID_ARG;
    }
    if (m->v.rows != m->v.cols) {
        mf::set_last_error("mf_residual_norm_noalloc: matrix is %d x %d, a square system is required", m->v.rows,
                           m->v.cols);
        return MF_ERR_INVALID_ARG;
    }
    if (m->v.tilem > MF_NOALLOC_MAX_STRIPS) {
        mf::set_last_error(
            "mf_residual_norm_noalloc: %d rows exceed the fixed scratch limit of %d rows (%d strips of 16); use "
            "mf_residual_norm",
            m->v.rows, MF_NOALLOC_MAX_STRIPS * MF_TILE, MF_NOALLOC_MAX_STRIPS);
        return MF_ERR_INVALID_ARG;
    }
    double *part = nullptr;
    MF_TRY(scratch_address(m->device, &part));
    return mf::residual_norm(m->v, b, x, part, out, (cudaStream_t)stream);
}
