// residual.cu -- FP64 true relative residual ||b - A x|| / ||b||.
//
// The reference checks every solve on the host with a tiled FP64 product and
// sequential sums (src/main-cg.cu:978-1011, 1543-1576).  Here one kernel
// computes, per 16-row strip, the rows of A x in blockspmv_cpu's summation
// order, the squared residual and the squared right-hand side of the strip
// (a fixed 16-lane tree), and writes the two strip partials; a second kernel
// sums the strip partials in a fixed order.  The result is the same on every
// run, whatever the launch shape.
#include "spmv_core.cuh"

namespace mf {

// Per-strip partials: part[2 s] = sum over the strip of (b - A x)^2,
// part[2 s + 1] = sum of b^2.
__global__ void __launch_bounds__(256) k_resid_strips(MfTiles A, const double *__restrict__ b,
                                                      const double *__restrict__ x, double *__restrict__ part)
{
    const int r = threadIdx.x & 15;
    for (int s = blockIdx.x * 16 + (threadIdx.x >> 4); s < A.tilem; s += gridDim.x * 16) {
        const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
        double d2 = 0.0, b2 = 0.0;
        if (r < rowlen) {
            const int i = s * MF_TILE + r;
            const double d = b[i] - row_fp64(A, s, r, rowlen, x);
            d2 = d * d;
            b2 = b[i] * b[i];
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            d2 += __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), d2, o, 16);
            b2 += __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), b2, o, 16);
        }
        if (r == 0) {
            part[2 * s] = d2;
            part[2 * s + 1] = b2;
        }
    }
}

// One CTA: thread k sums strips [k*per, (k+1)*per) in order, then a fixed
// tree over the threads.  out[0] = relative residual, out[1] = ||b - A x||,
// out[2] = ||b||.
__global__ void __launch_bounds__(1024) k_resid_reduce(int nstrips, const double *__restrict__ part,
                                                       double *__restrict__ out)
{
    __shared__ double s_warp[32];
    const int per = (nstrips + 1023) / 1024;
    const int a = threadIdx.x * per, e = min(nstrips, a + per);
    double d2 = 0.0, b2 = 0.0;
    for (int s = a; s < e; s++) {
        d2 += part[2 * s];
        b2 += part[2 * s + 1];
    }
    d2 = block_sum<1024>(d2, s_warp);
    b2 = block_sum<1024>(b2, s_warp);
    if (threadIdx.x == 0) {
        const double rn = sqrt(d2), bn = sqrt(b2);
        out[0] = bn > 0.0 ? rn / bn : rn;
        out[1] = rn;
        out[2] = bn;
    }
}

mf_status residual_norm(const MfTiles &A, const double *b, const double *x, double *part, double *out,
                        cudaStream_t s)
{
    if (A.tilem > 0) {
        int grid = ceil_div(A.tilem, 16);
        if (grid > 148 * 8) grid = 148 * 8;
        k_resid_strips<<<grid, 256, 0, s>>>(A, b, x, part);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    k_resid_reduce<<<1, 1024, 0, s>>>(A.tilem, part, out);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

}  // namespace mf

using namespace mf;

extern "C" mf_status mf_residual_norm(mf_matrix m, const double *b, const double *x, double *out, void *stream)
{
    if (!m || !b || !x || !out) {
        set_last_error("mf_residual_norm: null argument");
        return MF_ERR_INVALID_ARG;
    }
    if (m->v.rows != m->v.cols) {
        set_last_error("mf_residual_norm: matrix is %d x %d, a square system is required", m->v.rows, m->v.cols);
        return MF_ERR_INVALID_ARG;
    }
    const size_t need = sizeof(double) * 2 * (size_t)(m->v.tilem > 0 ? m->v.tilem : 1);
    if (m->resid_bytes < need) {
        if (m->d_resid) cudaFree(m->d_resid);
        m->d_resid = nullptr;
        m->resid_bytes = 0;
        MF_CUDA(cudaMalloc(&m->d_resid, need));
        m->resid_bytes = need;
    }
    return residual_norm(m->v, b, x, m->d_resid, out, (cudaStream_t)stream);
}
