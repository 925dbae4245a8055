// spmv_core.cuh -- per-row tiled SpMV building blocks shared by the SpMV and
// solver kernels.
//
// One thread owns one row of a 16-row strip (a tile-row).  It walks the
// strip's tiles in column order; inside a tile it sums its row's entries
// sequentially, then adds the tile's partial to the row total.  This is the
// summation order of the reference's blockspmv_cpu (src/blockspmv_cpu.h:98-108),
// and products and sums are rounded separately (no FMA contraction), so the
// FP64 result is bit-identical to that CPU code.
#pragma once
#include <cuda_fp16.h>

#include "mf_internal.h"

namespace mf {

// In-tile row bounds [lo, hi) of row r of tile t.
__device__ __forceinline__ void tile_row_bounds(const MfTiles &A, int t, int r, int rowlen, int off, int nz,
                                                int &lo, int &hi)
{
    const int po = A.rows_multiple_of_16 ? t * MF_TILE : A.csrptr_offset[t];
    lo = A.ptr[po + r];
    hi = (r == rowlen - 1) ? nz : (int)A.ptr[po + r + 1];
}

// FP64 row of strip `bi` against x (reference order, no contraction).  The
// next tile's metadata (entry offset, column, in-tile row bounds) is loaded
// before the current tile's entries are summed, so its latency overlaps the
// current tile's gathers of x.
__device__ __forceinline__ double row_fp64(const MfTiles &A, int bi, int r, int rowlen, const double *__restrict__ x)
{
    double y = 0.0;
    const int t0 = A.tile_ptr[bi], t1 = A.tile_ptr[bi + 1];
    if (t0 >= t1) return y;
    int off = A.tile_nnz[t0];
    int nxt = A.tile_nnz[t0 + 1];
    int xo = A.tile_columnidx[t0] * MF_TILE;
    int lo, hi;
    tile_row_bounds(A, t0, r, rowlen, off, nxt - off, lo, hi);
    for (int t = t0; t < t1; t++) {
        int nxt2 = nxt, xo2 = 0, lo2 = 0, hi2 = 0;
        if (t + 1 < t1) {
            nxt2 = A.tile_nnz[t + 2];
            xo2 = A.tile_columnidx[t + 1] * MF_TILE;
            tile_row_bounds(A, t + 1, r, rowlen, nxt, nxt2 - nxt, lo2, hi2);
        }
        double s = 0.0;
        for (int k = off + lo; k < off + hi; k++) s = __dadd_rn(s, __dmul_rn(x[xo + A.col[k]], A.val[k]));
        y = __dadd_rn(y, s);
        off = nxt;
        nxt = nxt2;
        xo = xo2;
        lo = lo2;
        hi = hi2;
    }
    return y;
}

}  // namespace mf
