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

}  // namespace

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
