// spmv.cu -- standalone FP64 tiled SpMV (the role of the reference's
// stir_spmv_cuda_kernel_newcsr, src/Mille-feuille-cg.h:97-166, and of
// blockspmv_cpu, src/blockspmv_cpu.h:2-112).  Thread per row; no atomics;
// bit-identical to blockspmv_cpu.
#include "spmv_core.cuh"

namespace mf {
namespace {

constexpr int SPMV_NT = 256;

__global__ void __launch_bounds__(SPMV_NT) k_spmv_fp64(MfTiles A, const double *__restrict__ x, double *__restrict__ y)
{
    const int strips_per_cta = SPMV_NT / MF_TILE;
    for (int bi = blockIdx.x * strips_per_cta + (threadIdx.x >> 4); bi < A.tilem; bi += gridDim.x * strips_per_cta) {
        const int r = threadIdx.x & 15;
        const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
        if (r < rowlen) y[bi * MF_TILE + r] = row_fp64(A, bi, r, rowlen, x);
    }
}

// As k_spmv_fp64, with each entry's in-tile column read from the 4-bit
// packed array (two per byte, even positions in the high nibble), as
// blockspmv_cpu reads csr_compressedIdx (src/blockspmv_cpu.h:101-103).
__global__ void __launch_bounds__(SPMV_NT) k_spmv_fp64_cidx(MfTiles A, const unsigned char *__restrict__ cidx,
                                                             const double *__restrict__ x, double *__restrict__ y)
{
    const int strips_per_cta = SPMV_NT / MF_TILE;
    for (int bi = blockIdx.x * strips_per_cta + (threadIdx.x >> 4); bi < A.tilem; bi += gridDim.x * strips_per_cta) {
        const int r = threadIdx.x & 15;
        const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
        if (r >= rowlen) continue;
        double acc = 0.0;
        const int t0 = A.tile_ptr[bi], t1 = A.tile_ptr[bi + 1];
        int off = A.tile_nnz[t0];
        for (int t = t0; t < t1; t++) {
            const int nxt = A.tile_nnz[t + 1];
            const int xo = A.tile_columnidx[t] * MF_TILE;
            int lo, hi;
            tile_row_bounds(A, t, r, rowlen, off, nxt - off, lo, hi);
            double s = 0.0;
            for (int k = off + lo; k < off + hi; k++) {
                const unsigned char b = cidx[k >> 1];
                const int c = (k & 1) ? (b & 0x0F) : (b >> 4);
                s = __dadd_rn(s, __dmul_rn(x[xo + c], A.val[k]));
            }
            acc = __dadd_rn(acc, s);
            off = nxt;
        }
        y[bi * MF_TILE + r] = acc;
    }
}

}  // namespace

mf_status spmv_fp64_cidx(const MfTiles &A, const unsigned char *cidx, const double *x, double *y, cudaStream_t s)
{
    if (A.tilem == 0) return MF_OK;
    int grid = ceil_div(A.tilem, SPMV_NT / MF_TILE);
    k_spmv_fp64_cidx<<<grid, SPMV_NT, 0, s>>>(A, cidx, x, y);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

mf_status spmv_fp64(const MfTiles &A, const double *x, double *y, cudaStream_t s)
{
    if (A.tilem == 0) return MF_OK;
    int grid = ceil_div(A.tilem, SPMV_NT / MF_TILE);
    k_spmv_fp64<<<grid, SPMV_NT, 0, s>>>(A, x, y);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

}  // namespace mf
