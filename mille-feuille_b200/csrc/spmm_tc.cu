// spmm_tc.cu -- Y = A X for k <= 16 columns with the dense tiles on the
// tensor cores: FP16 inputs, FP32 accumulation (mf_spmm_f16).
//
// No reference counterpart: the reference runs one SpMV per vector
// (src/Mille-feuille-cg.h:97-166).  A 16x16 tile with at least `fill`
// entries is kept as a dense FP16 block (built once per matrix and fill
// threshold, duplicates added in FP32 before the rounding); a warp owns a
// 16-row strip and multiplies each dense tile of it by the matching 16-row
// block of X with two mma.sync m16n8k16 instructions (columns 0-7 and
// 8-15), the accumulators held in the MMA fragment layout; the strip's
// sparse tiles are added by the same threads into the same accumulators
// (each thread owns rows gid and gid + 8 and four columns), with FP32
// values.  X is first scaled per column by a power of two that maps its
// largest magnitude to [0.5, 1] and rounded to FP16 (row-major, 16 halves
// per row); Y is rescaled and written in FP64.  Every output is summed in
// a fixed order (deterministic).  Accuracy: FP16 rounding of A's dense
// tiles and of X (2^-11 relative each), FP32 sums.
//
// The MMA is the warp-level form, which Blackwell runs on its tensor cores;
// a 16 x 16 x 16 block is far below the smallest tcgen05 tile (64 rows), so
// tcgen05 with TMEM accumulators would idle most of each instruction here.
#include <cuda_fp16.h>

#include <algorithm>

#include "mf_internal.h"
#include "spmv_core.cuh"

namespace mf {
namespace {

constexpr int TC_NT = 256;  // 8 warps per CTA, one strip per warp at a time

int tc_grid(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    return (int)(g < 1 ? 1 : g > 148 * 32 ? 148 * 32 : g);
}

__global__ void k_tc_mark(int T, const int *__restrict__ tile_nnz, const unsigned char *__restrict__ f16ok, int fill,
                          int *__restrict__ flag)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        flag[t] = (tile_nnz[t + 1] - tile_nnz[t] >= fill && (f16ok[t] & 1)) ? 1 : 0;
}

// index[t] = the dense block of tile t (the scan of the flags), or -1
__global__ void k_tc_index(int T, const int *__restrict__ flag, int *__restrict__ index)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        if (!flag[t]) index[t] = -1;
}

// One warp per dense tile: lane 0 adds the tile's entries (in entry order,
// duplicates summed) into a 16x16 FP32 block in shared memory, then the
// warp rounds it to FP16, row-major.
__global__ void __launch_bounds__(TC_NT) k_tc_fill(MfTiles A, int T, const int *__restrict__ tile_strip,
                                                   const int *__restrict__ index, __half *__restrict__ dense)
{
    __shared__ float blk[TC_NT / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *b = blk[w];
    for (int t = blockIdx.x * (TC_NT / 32) + w; t < T; t += gridDim.x * (TC_NT / 32)) {
        const int di = index[t];
        if (di < 0) continue;  // uniform over the warp
        for (int i = lane; i < 256; i += 32) b[i] = 0.f;
        __syncwarp();
        if (lane == 0) {
            const int bi = tile_strip[t];
            const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
            const int off = A.tile_nnz[t], nz = A.tile_nnz[t + 1] - off;
            for (int r = 0; r < rowlen; r++) {
                int lo, hi;
                tile_row_bounds(A, t, r, rowlen, off, nz, lo, hi);
                for (int e = off + lo; e < off + hi; e++) b[r * 16 + A.col[e]] += (float)A.val[e];
            }
        }
        __syncwarp();
        for (int i = lane; i < 256; i += 32) dense[(size_t)di * 256 + i] = __float2half_rn(b[i]);
        __syncwarp();
    }
}

// Per column j < k: the largest |X[:, j]| (float bits; atomicMax on
// non-negative floats orders like the values).  Each thread keeps the
// maxima of its rows, the block combines them (warp shuffles, then shared
// memory), one atomic per block and column.
__global__ void __launch_bounds__(256) k_tc_colmax(int n, int k, const double *__restrict__ X, int ldx,
                                                   unsigned *__restrict__ mx)
{
    __shared__ float s_m[8][16];
    float m[16];
#pragma unroll
    for (int j = 0; j < 16; j++) m[j] = 0.f;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
#pragma unroll
        for (int j = 0; j < 16; j++)
            if (j < k) m[j] = fmaxf(m[j], (float)fabs(X[(size_t)j * ldx + r]));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        float v = m[j];
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) s_m[w][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < 16 && (int)threadIdx.x < k) {
        float v = 0.f;
        for (int ww = 0; ww < 8; ww++) v = fmaxf(v, s_m[ww][threadIdx.x]);
        atomicMax(&mx[threadIdx.x], __float_as_uint(v));
    }
}

// scale[j] = 2^-e with 2^(e-1) <= max|X[:, j]| < 2^e (1 for a zero column),
// exact powers of two; inv[j] = 1 / scale[j]
__global__ void k_tc_scale(int k, const unsigned *__restrict__ mx, float *__restrict__ scale, float *__restrict__ inv)
{
    const int j = threadIdx.x;
    if (j < 16) {
        const float m = j < k ? __uint_as_float(mx[j]) : 0.f;
        int e = 0;
        if (m > 0.f) frexpf(m, &e);
        scale[j] = ldexpf(1.f, -e);
        inv[j] = ldexpf(1.f, e);
    }
}

// X scaled per column and rounded to FP16, row-major with 16 halves per
// row (one thread per row: column-major X read coalesced column by column),
// rows up to the padded column count, columns >= k zero
__global__ void k_tc_xpack(int nrow_pad, int n, int k, const double *__restrict__ X, int ldx,
                           const float *__restrict__ scale, __half *__restrict__ x16)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrow_pad; r += gridDim.x * blockDim.x) {
        unsigned w[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
            const float v0 = (j < k && r < n) ? (float)(X[(size_t)j * ldx + r] * (double)scale[j]) : 0.f;
            const float v1 = (j + 1 < k && r < n) ? (float)(X[(size_t)(j + 1) * ldx + r] * (double)scale[j + 1]) : 0.f;
            w[j / 2] = (unsigned)__half_as_ushort(__float2half_rn(v0)) |
                       ((unsigned)__half_as_ushort(__float2half_rn(v1)) << 16);
        }
        uint4 *d = reinterpret_cast<uint4 *>(x16 + (size_t)r * 16);
        d[0] = make_uint4(w[0], w[1], w[2], w[3]);
        d[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

__device__ __forceinline__ unsigned pack_h2(__half lo, __half hi)
{
    return (unsigned)__half_as_ushort(lo) | ((unsigned)__half_as_ushort(hi) << 16);
}

// D (16x8, FP32) += A (16x16, FP16, row-major fragments) * B (16x8, FP16)
__device__ __forceinline__ void mma_16816(float *d, unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                          unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One warp per strip.  Fragment layout of m16n8k16 (thread lane: gid =
// lane / 4, tig = lane % 4): A holds rows gid and gid + 8, columns 2 tig,
// 2 tig + 1 and the same + 8; B holds rows 2 tig, 2 tig + 1 (+ 8) of column
// gid; D holds rows gid, gid + 8 and columns 2 tig, 2 tig + 1.
template <bool TWO>
__global__ void __launch_bounds__(TC_NT) k_spmm_tc(MfTiles A, const int *__restrict__ index,
                                                   const __half *__restrict__ dense, const __half *__restrict__ x16,
                                                   int k, const float *__restrict__ inv, double *__restrict__ Y,
                                                   int ldy)
{
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int nwarp = gridDim.x * (TC_NT / 32);
    for (int bi = blockIdx.x * (TC_NT / 32) + (threadIdx.x >> 5); bi < A.tilem; bi += nwarp) {
        const int rowlen = (bi == A.tilem - 1) ? A.rows - bi * MF_TILE : MF_TILE;
        float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
        const int t0 = A.tile_ptr[bi], t1 = A.tile_ptr[bi + 1];
        // the next tile's metadata (dense index, column, entry offsets) is
        // loaded before the current tile is computed
        int di = t0 < t1 ? index[t0] : -1, xo = t0 < t1 ? A.tile_columnidx[t0] * MF_TILE : 0;
        int off = A.tile_nnz[t0], nxt = t0 < t1 ? A.tile_nnz[t0 + 1] : off;
        for (int t = t0; t < t1; t++) {  // uniform over the warp
            int di2 = -1, xo2 = 0, nxt2 = nxt;
            if (t + 1 < t1) {
                di2 = index[t + 1];
                xo2 = A.tile_columnidx[t + 1] * MF_TILE;
                nxt2 = A.tile_nnz[t + 2];
            }
            const __half *xb = x16 + (size_t)xo * 16;
            if (di >= 0) {
                const __half *a = dense + (size_t)di * 256;
                const unsigned a0 = *reinterpret_cast<const unsigned *>(a + gid * 16 + 2 * tig);
                const unsigned a1 = *reinterpret_cast<const unsigned *>(a + (gid + 8) * 16 + 2 * tig);
                const unsigned a2 = *reinterpret_cast<const unsigned *>(a + gid * 16 + 2 * tig + 8);
                const unsigned a3 = *reinterpret_cast<const unsigned *>(a + (gid + 8) * 16 + 2 * tig + 8);
                {
                    const __half *xc = xb + gid;
                    mma_16816(d0, a0, a1, a2, a3, pack_h2(xc[(2 * tig) * 16], xc[(2 * tig + 1) * 16]),
                              pack_h2(xc[(2 * tig + 8) * 16], xc[(2 * tig + 9) * 16]));
                }
                if (TWO) {
                    const __half *xc = xb + 8 + gid;
                    mma_16816(d1, a0, a1, a2, a3, pack_h2(xc[(2 * tig) * 16], xc[(2 * tig + 1) * 16]),
                              pack_h2(xc[(2 * tig + 8) * 16], xc[(2 * tig + 9) * 16]));
                }
            } else {
                // sparse tile: rows gid and gid + 8, this thread's columns
                const int nz = nxt - off;
                for (int h = 0; h < 2; h++) {
                    const int r = gid + 8 * h;
                    if (r >= rowlen) continue;
                    int lo, hi;
                    tile_row_bounds(A, t, r, rowlen, off, nz, lo, hi);
                    for (int e = off + lo; e < off + hi; e++) {
                        const float v = A.val_low[e];
                        const __half *xr = xb + (size_t)A.col[e] * 16;
                        d0[2 * h] = fmaf(v, __half2float(xr[2 * tig]), d0[2 * h]);
                        d0[2 * h + 1] = fmaf(v, __half2float(xr[2 * tig + 1]), d0[2 * h + 1]);
                        if (TWO) {
                            d1[2 * h] = fmaf(v, __half2float(xr[8 + 2 * tig]), d1[2 * h]);
                            d1[2 * h + 1] = fmaf(v, __half2float(xr[9 + 2 * tig]), d1[2 * h + 1]);
                        }
                    }
                }
            }
            di = di2;
            xo = xo2;
            off = nxt;
            nxt = nxt2;
        }
        for (int h = 0; h < 2; h++) {
            const int r = gid + 8 * h;
            if (r >= rowlen) continue;
            const size_t i = (size_t)bi * MF_TILE + r;
            const int c0 = 2 * tig, c1 = 2 * tig + 1, c2 = 8 + 2 * tig, c3 = 9 + 2 * tig;
            if (c0 < k) Y[(size_t)c0 * ldy + i] = (double)(d0[2 * h] * inv[c0]);
            if (c1 < k) Y[(size_t)c1 * ldy + i] = (double)(d0[2 * h + 1] * inv[c1]);
            if (TWO && c2 < k) Y[(size_t)c2 * ldy + i] = (double)(d1[2 * h] * inv[c2]);
            if (TWO && c3 < k) Y[(size_t)c3 * ldy + i] = (double)(d1[2 * h + 1] * inv[c3]);
        }
    }
}

// Dense blocks for threshold `fill` (kept on the handle; rebuilt when the
// threshold changes)
mf_status tc_prepare(mf_matrix m, int fill, cudaStream_t s)
{
    if (m->d_tc_index && m->tc_fill == fill) return MF_OK;
    const int T = m->v.tilenum;
    if (m->d_tc_index) cudaFree(m->d_tc_index);
    if (m->d_tc_dense) cudaFree(m->d_tc_dense);
    m->d_tc_index = nullptr;
    m->d_tc_dense = nullptr;
    m->tc_fill = 0;
    m->tc_ndense = 0;
    MF_CUDA(cudaMalloc(&m->d_tc_index, sizeof(int) * (size_t)(T + 1) + 16));
    int *flag = nullptr;
    MF_CUDA(pool_malloc_async(&flag, sizeof(int) * (size_t)(T + 1) + 16, s));
    int nd = 0;
    if (T > 0) {
        k_tc_mark<<<tc_grid(T, 256), 256, 0, s>>>(T, m->d_tile_nnz, m->d_f16ok, fill, flag);
        note_launch();
        MF_CUDA(cudaGetLastError());
        MF_TRY(exclusive_scan_i32(flag, m->d_tc_index, T, s, &nd));
        k_tc_index<<<tc_grid(T, 256), 256, 0, s>>>(T, flag, m->d_tc_index);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    cudaFreeAsync(flag, s);
    MF_CUDA(cudaMalloc(&m->d_tc_dense, sizeof(__half) * 256 * (size_t)(nd > 0 ? nd : 1)));
    if (nd > 0) {
        k_tc_fill<<<tc_grid((long long)T * 32, TC_NT), TC_NT, 0, s>>>(m->v, T, m->d_tile_rowidx, m->d_tc_index,
                                                                       (__half *)m->d_tc_dense);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    m->tc_fill = fill;
    m->tc_ndense = nd;
    return MF_OK;
}

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" mf_status mf_spmm_f16(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, int dense_fill,
                                 int *dense_tiles, void *stream)
{
    if (!m || k < 1 || k > 16 || dense_fill > 256 || (m->v.rows > 0 && (!X || !Y)) || ldx < m->v.cols ||
        ldy < m->v.rows) {
        set_last_error("mf_spmm_f16: null argument, k = %d outside 1..16, fill above 256 or a short leading dimension",
                       k);
        return MF_ERR_INVALID_ARG;
    }
    const int fill = dense_fill > 0 ? dense_fill : 64;
    cudaStream_t s = (cudaStream_t)stream;
    MF_TRY(tc_prepare(m, fill, s));
    if (dense_tiles) *dense_tiles = m->tc_ndense;
    if (m->v.rows == 0) return MF_OK;
    const int nrow_pad = m->v.tilen * MF_TILE;
    __half *x16 = nullptr;  // 32 bytes per row: 16-byte aligned rows
    MF_CUDA(pool_malloc_async(&x16, sizeof(__half) * 16 * (size_t)nrow_pad + 256, s));
    unsigned *mx = (unsigned *)(x16 + 16 * (size_t)nrow_pad);
    float *scale = (float *)(mx + 16), *inv = scale + 16;
    MF_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned) * 16, s));
    if (m->v.cols > 0) {
        // a resident wave of blocks, each striding over the rows
        k_tc_colmax<<<std::min(tc_grid(m->v.cols, 256), 148 * 4), 256, 0, s>>>(m->v.cols, k, X, ldx, mx);
        note_launch();
    }
    k_tc_scale<<<1, 32, 0, s>>>(k, mx, scale, inv);
    note_launch();
    k_tc_xpack<<<tc_grid(nrow_pad, 256), 256, 0, s>>>(nrow_pad, m->v.cols, k, X, ldx, scale, x16);
    note_launch();
    const int grid = tc_grid((long long)m->v.tilem * 32, TC_NT);
    if (k > 8)
        k_spmm_tc<true><<<grid, TC_NT, 0, s>>>(m->v, m->d_tc_index, (const __half *)m->d_tc_dense, x16, k, inv, Y, ldy);
    else
        k_spmm_tc<false><<<grid, TC_NT, 0, s>>>(m->v, m->d_tc_index, (const __half *)m->d_tc_dense, x16, k, inv, Y,
                                                ldy);
    note_launch();
    MF_CUDA(cudaGetLastError());
    cudaFreeAsync(x16, s);
    return MF_OK;
}
