// tile_build.cu -- CSR -> 16x16 tile-CSR conversion on the GPU.
//
// Produces, bit-exact, the arrays of the reference Tile_create
// (src/csr2block.h:267-422): tiles of a tile-row in ascending column order,
// entries of a tile in CSR order, u8 in-tile row pointers (wrapping mod 256
// as the reference's unsigned char arithmetic does).  Then the derived
// arrays of the reference host drivers: the non-empty-row lists
// (src/main-cg.cu:1231-1288), the blockspmv_cpu row-block schedule
// (src/blockspmv_cpu.h:35-83), and the per-class payloads
// (src/main-cg-mixed.cu:2325-2342).
//
// Design (not the reference's): one CTA per tile-row sorts the tile-row's
// entries by (tile column, CSR position) with a bitonic network in shared
// memory (global memory for tile-rows above SORT_CAP entries).  After one
// scan of tile counts, a second pass scatters: because tiles are ordered by
// column and entries keep CSR order, an entry's destination is simply the
// tile-row's first CSR offset plus its sorted position, so values move in one
// coalesced pass with no per-entry search.
#include <cuda_fp16.h>

#include "mf_internal.h"

namespace mf {
namespace {

constexpr int BUILD_NT = 256;
constexpr int SORT_CAP = 4096;  // entries sorted in shared memory
constexpr unsigned long long KEY_PAD = ~0ull;

// Ascending bitonic network over P (power of two) keys; only pairs whose
// partner index is above the lower index are compared, so virtual +inf
// padding beyond m never moves.  `keys` is shared or global memory.
__device__ void bitonic_sort(unsigned long long *keys, int m, int P)
{
    for (int k = 2; k <= P; k <<= 1) {
        const int half = k >> 1;
        for (int q = threadIdx.x; q < P / 2; q += blockDim.x) {
            int i = (q / half) * k + (q % half);
            int j = i ^ (k - 1);
            if (j < m) {
                unsigned long long a = keys[i], b = keys[j];
                if (a > b) { keys[i] = b; keys[j] = a; }
            }
        }
        __syncthreads();
        for (int jj = half >> 1; jj > 0; jj >>= 1) {
            for (int q = threadIdx.x; q < P / 2; q += blockDim.x) {
                int i = (q / jj) * (2 * jj) + (q % jj);
                int j = i + jj;
                if (j < m) {
                    unsigned long long a = keys[i], b = keys[j];
                    if (a > b) { keys[i] = b; keys[j] = a; }
                }
            }
            __syncthreads();
        }
    }
}

// Pass 1: sort each tile-row's entries by (tile column, CSR position); write
// the permutation and the number of distinct tile columns.
__global__ void __launch_bounds__(BUILD_NT)
k_sort_tilerows(int tilem, int rowA, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                int *__restrict__ perm, unsigned long long *__restrict__ big_keys, int *__restrict__ tilecnt)
{
    __shared__ unsigned long long s_keys[SORT_CAP];
    __shared__ int s_cnt[BUILD_NT / 32];
    for (int bi = blockIdx.x; bi < tilem; bi += gridDim.x) {
        const int rs = bi * MF_TILE, re = min(rowA, rs + MF_TILE);
        const int base = rowptr[rs], m = rowptr[re] - base;
        int P = 1;
        while (P < m) P <<= 1;
        unsigned long long *keys = (m <= SORT_CAP) ? s_keys : (big_keys + base);
        if (m <= SORT_CAP) {
            for (int k = threadIdx.x; k < P; k += BUILD_NT)
                s_keys[k] = (k < m) ? (((unsigned long long)(colidx[base + k] >> 4) << 32) | (unsigned)k) : KEY_PAD;
        } else {
            for (int k = threadIdx.x; k < m; k += BUILD_NT)
                keys[k] = ((unsigned long long)(colidx[base + k] >> 4) << 32) | (unsigned)k;
        }
        __syncthreads();
        bitonic_sort(keys, m, P);
        int cnt = 0;
        for (int k = threadIdx.x; k < m; k += BUILD_NT) {
            unsigned long long key = keys[k];
            perm[base + k] = (int)(key & 0xffffffffull);
            if (k == 0 || (keys[k - 1] >> 32) != (key >> 32)) cnt++;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if ((threadIdx.x & 31) == 0) s_cnt[threadIdx.x >> 5] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < BUILD_NT / 32; w++) t += s_cnt[w];
            tilecnt[bi] = t;
        }
        __syncthreads();
    }
}

// Pass 2: scatter entries to tile order; tile columns, tile offsets, the
// first position of each non-empty (tile,row) run, tile row index.
__global__ void __launch_bounds__(BUILD_NT)
k_fill_tilerows(int tilem, int rowA, int rp0, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                const double *__restrict__ val, const float *__restrict__ val_low, const int *__restrict__ perm,
                const int *__restrict__ tile_ptr, int *__restrict__ tile_columnidx, int *__restrict__ tile_nnz,
                int *__restrict__ tile_rowidx, int *__restrict__ run_start, double *__restrict__ out_val,
                float *__restrict__ out_low, unsigned char *__restrict__ out_col)
{
    __shared__ int s_rp[MF_TILE + 1];
    __shared__ int s_warp[BUILD_NT / 32];
    __shared__ int s_carry;
    for (int bi = blockIdx.x; bi < tilem; bi += gridDim.x) {
        const int rs = bi * MF_TILE, re = min(rowA, rs + MF_TILE), rows = re - rs;
        if (threadIdx.x <= rows) s_rp[threadIdx.x] = rowptr[rs + threadIdx.x];
        if (threadIdx.x == 0) s_carry = 0;
        __syncthreads();
        const int base = s_rp[0], m = s_rp[rows] - base;
        const int t0 = tile_ptr[bi];
        for (int c0 = 0; c0 < m; c0 += BUILD_NT) {
            const int k = c0 + threadIdx.x;
            int src = 0, jc = -1, row = 0, head = 0, rowhead = 0;
            if (k < m) {
                src = base + perm[base + k];
                jc = colidx[src] >> 4;
                // row of src: last r with s_rp[r] <= src
                int lo = 0, hi = rows - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (s_rp[mid] <= src) lo = mid; else hi = mid - 1;
                }
                row = lo;
                if (k == 0) {
                    head = 1;
                    rowhead = 1;
                } else {
                    int psrc = base + perm[base + k - 1];
                    int pjc = colidx[psrc] >> 4;
                    head = (pjc != jc);
                    if (head) rowhead = 1;
                    else {
                        int plo = 0, phi = rows - 1;
                        while (plo < phi) {
                            int mid = (plo + phi + 1) >> 1;
                            if (s_rp[mid] <= psrc) plo = mid; else phi = mid - 1;
                        }
                        rowhead = (plo != row);
                    }
                }
            }
            // inclusive scan of head flags across the CTA -> tile ordinal
            int x = head;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_warp[w] = x;
            __syncthreads();
            int woff = 0, tot = 0;
            for (int i = 0; i < BUILD_NT / 32; i++) {
                if (i < w) woff += s_warp[i];
                tot += s_warp[i];
            }
            const int ord = s_carry + woff + x - 1;  // tile ordinal of this entry
            if (k < m) {
                const int t = t0 + ord;
                const int dst = base - rp0 + k;
                if (head) {
                    tile_columnidx[t] = jc;
                    tile_nnz[t] = dst;
                    tile_rowidx[t] = bi;
                }
                if (rowhead) run_start[(size_t)t * MF_TILE + row] = dst;  // absolute position
                out_val[dst] = val[src];
                out_low[dst] = val_low ? val_low[src] : (float)val[src];
                out_col[dst] = (unsigned char)(colidx[src] & 15);
            }
            __syncthreads();
            if (threadIdx.x == 0) s_carry += tot;
            __syncthreads();
        }
        __syncthreads();
    }
}

// Per tile: in-tile u8 row pointers from the first position of each
// non-empty row (empty rows take the start of the next non-empty row, as an
// exclusive scan of per-row counts does), u8 entry count, row-pointer offset,
// and the non-empty-row count with the reference's test (stop != start,
// src/main-cg.cu:1241-1245).
__global__ void k_tile_finish(int tilem, int rowA, int T, const int *__restrict__ tile_ptr,
                              const int *__restrict__ tile_rowidx, int *__restrict__ tile_nnz,
                              const int *__restrict__ run_start, int *__restrict__ csrptr_offset,
                              unsigned char *__restrict__ blkptr, unsigned char *__restrict__ blknnznnz,
                              int *__restrict__ nz_rows, int *__restrict__ err, int nnz_total)
{
    const int last_row_tiles_begin = (tilem > 0) ? tile_ptr[tilem - 1] : 0;
    const int rowlen_last = rowA - (tilem - 1) * MF_TILE;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int off = tile_nnz[t];
        const int nz = ((t + 1 < T) ? tile_nnz[t + 1] : nnz_total) - off;
        if (nz > 256) atomicExch(err, (int)MF_ERR_UNSUPPORTED);
        const int bi = tile_rowidx[t];
        const int rowlen = (bi == tilem - 1) ? rowlen_last : MF_TILE;
        const int po = (t < last_row_tiles_begin) ? t * MF_TILE
                                                   : last_row_tiles_begin * MF_TILE + (t - last_row_tiles_begin) * rowlen_last;
        csrptr_offset[t] = po;
        blknnznnz[t] = (unsigned char)nz;
        int next = nz, nonempty = 0;
        unsigned char p8[MF_TILE];
        for (int r = rowlen - 1; r >= 0; r--) {
            const int st = run_start[(size_t)t * MF_TILE + r];
            if (st >= 0) next = st - off;
            if (r == 0) next = 0;
            p8[r] = (unsigned char)next;
        }
        for (int r = 0; r < rowlen; r++) {
            blkptr[po + r] = p8[r];
            const int stop = (r == rowlen - 1) ? nz : (int)p8[r + 1];
            if (stop != (int)p8[r]) nonempty++;
        }
        nz_rows[t] = 1 + nonempty;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        tile_nnz[T] = nnz_total;
        csrptr_offset[T] = (T > last_row_tiles_begin) ? last_row_tiles_begin * MF_TILE + (T - last_row_tiles_begin) * rowlen_last
                                                      : T * MF_TILE;
        blknnznnz[T] = 0;
    }
}

// Non-empty-row lists (src/main-cg.cu:1262-1288): per tile a sentinel
// (row 0, offset 0) then (row, u8 end offset) for every non-empty row.
__global__ void k_nonzero_lists(int tilem, int rowA, int T, const int *__restrict__ tile_rowidx,
                                const int *__restrict__ tile_nnz, const int *__restrict__ csrptr_offset,
                                const unsigned char *__restrict__ blkptr, const int *__restrict__ nzr,
                                unsigned char *__restrict__ rowid, unsigned char *__restrict__ ptrnew)
{
    const int rowlen_last = rowA - (tilem - 1) * MF_TILE;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int rowlen = (tile_rowidx[t] == tilem - 1) ? rowlen_last : MF_TILE;
        const int nz = tile_nnz[t + 1] - tile_nnz[t];
        const int po = csrptr_offset[t];
        int o = nzr[t];
        rowid[o] = 0;
        ptrnew[o] = 0;
        o++;
        for (int r = 0; r < rowlen; r++) {
            int stop = (r == rowlen - 1) ? nz : blkptr[po + r + 1];
            if (stop != blkptr[po + r]) {
                rowid[o] = (unsigned char)r;
                ptrnew[o] = (unsigned char)stop;
                o++;
            }
        }
    }
}

// Row-block schedule of blockspmv_cpu (src/blockspmv_cpu.h:35-83).
__global__ void k_rbb_count(int tilem, const int *__restrict__ tile_ptr, int *__restrict__ cnt,
                            int *__restrict__ block_signal)
{
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi <= tilem; bi += gridDim.x * blockDim.x) {
        if (bi == tilem) {
            cnt[bi] = 0;
            block_signal[bi] = 0;
            continue;
        }
        int k = tile_ptr[bi + 1] - tile_ptr[bi];
        cnt[bi] = (k <= 4) ? 1 : (k + 3) / 4;
        block_signal[bi] = k;
    }
}

__global__ void k_rbb_fill(int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ off,
                           unsigned *__restrict__ rowidx, int *__restrict__ cs, int *__restrict__ ce)
{
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < tilem; bi += gridDim.x * blockDim.x) {
        int k = tile_ptr[bi + 1] - tile_ptr[bi];
        int e = off[bi];
        if (k <= 4) {
            rowidx[e] = (unsigned)bi;
            cs[e] = 0;
            ce[e] = 0;
            continue;
        }
        int parts = (k + 3) / 4;
        int len = (k + parts - 1) / parts;
        for (int p = 0; p < parts; p++) {
            rowidx[e + p] = (unsigned)bi | 0x80000000u;
            cs[e + p] = tile_ptr[bi] + p * len;
            ce[e + p] = (p == parts - 1) ? tile_ptr[bi] + k : tile_ptr[bi] + (p + 1) * len;
        }
    }
}

// Static (value-range) class per tile: the smallest format that holds every
// value of the tile exactly.
//   int8 : every value an integer in [-128, 127]
//   fp16 : every value exactly representable in binary16
//   fp32 : every value exactly representable in binary32
//   fp64 : otherwise
// Payloads: fp16 = (half)(float)v, int8 = (int8_t)v (low byte of the
// truncated 32-bit integer), as src/main-cg-mixed.cu:2333-2336 builds them.
// f16ok: bit 0 every FP16 payload value of the tile is finite (|v| within
// binary16's range), the condition for running an inexact tile in FP16;
// bit 1 every nonzero one is also normal (|v| >= 2^-14: no subnormal loss).
__global__ void k_payloads(int T, const int *__restrict__ tile_nnz, const double *__restrict__ val,
                           const float *__restrict__ low, uint16_t *__restrict__ f16, int8_t *__restrict__ i8,
                           unsigned char *__restrict__ cls, unsigned char *__restrict__ f16ok,
                           int *__restrict__ class_count, int *__restrict__ max_nz)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int a = tile_nnz[t], b = tile_nnz[t + 1];
        bool is_int8 = true, in16 = true, in32 = true, fin16 = true, norm16 = true;
        for (int k = a; k < b; k++) {
            const double v = val[k];
            const double av = fabs(v);
            const half h = __float2half_rn(low[k]);
            f16[k] = __half_as_ushort(h);
            long long w = (av < 2147483648.0) ? (long long)__double2int_rz(v) : (long long)INT_MIN;
            i8[k] = (int8_t)(unsigned char)(unsigned)(int)w;
            if (!(v == trunc(v) && v >= -128.0 && v <= 127.0)) is_int8 = false;
            const float vf = (float)v;
            if ((double)vf != v) in32 = false;
            if ((double)__half2float(h) != v) in16 = false;
            if (__hisinf(h) || __hisnan(h)) fin16 = false;
            const unsigned short hb = __half_as_ushort(h);
            if (v != 0.0 && (hb & 0x7C00u) == 0) norm16 = false;  // zero or subnormal from a nonzero value
        }
        f16ok[t] = (unsigned char)((fin16 ? 1 : 0) | (fin16 && norm16 ? 2 : 0));
        unsigned char c = is_int8 ? MF_CLASS_INT8 : in16 ? MF_CLASS_FP16 : in32 ? MF_CLASS_FP32 : MF_CLASS_FP64;
        cls[t] = c;
        atomicAdd(&class_count[c], 1);
        atomicMax(max_nz, b - a);
    }
}

__global__ void k_validate(int rowA, int colA, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                           int *__restrict__ err)
{
    const int rp0 = rowptr[0], rpn = rowptr[rowA];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)rowA + (rpn - rp0);
         i += (long long)gridDim.x * blockDim.x) {
        if (i < rowA) {
            if (rowptr[i + 1] < rowptr[i]) atomicExch(err, (int)MF_ERR_INVALID_ARG);
        } else {
            int c = colidx[rp0 + (i - rowA)];
            if (c < 0 || c >= colA) atomicExch(err, (int)MF_ERR_INVALID_ARG);
        }
    }
}

// Strip partition: split tile-rows into `ctas` contiguous ranges of about
// equal cost (entries + 8 per tile + 16 per tile-row).
__global__ void k_strip_cost(int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ tile_nnz,
                             int *__restrict__ cost)
{
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi <= tilem; bi += gridDim.x * blockDim.x) {
        if (bi == tilem) { cost[bi] = 0; continue; }
        int t0 = tile_ptr[bi], t1 = tile_ptr[bi + 1];
        cost[bi] = (tile_nnz[t1] - tile_nnz[t0]) + 8 * (t1 - t0) + 16;
    }
}

__global__ void k_strip_split(int tilem, int ctas, const int *__restrict__ pref, int *__restrict__ part)
{
    const long long total = pref[tilem];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= ctas; g += gridDim.x * blockDim.x) {
        if (g == 0) { part[0] = 0; continue; }
        if (g == ctas) { part[g] = tilem; continue; }
        long long target = total * g / ctas;
        int lo = 0, hi = tilem;  // first bi with pref[bi] >= target
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (pref[mid] < target) lo = mid + 1; else hi = mid;
        }
        part[g] = lo;
    }
}

template <typename T>
mf_status dalloc(T **p, size_t n, size_t *acc)
{
    size_t bytes = sizeof(T) * (n > 0 ? n : 1) + 16;  // 16 B slack for vector loads at the tail
    MF_CUDA(cudaMalloc((void **)p, bytes));
    *acc += bytes;
    return MF_OK;
}

int grid_for(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

mf_status build_tiles(mf_matrix m, int rowA, int colA, const int *d_rowptr, const int *d_colidx,
                      const double *d_val, const float *d_val_low, cudaStream_t s)
{
    const int tilem = ceil_div(rowA, MF_TILE), tilen = ceil_div(colA, MF_TILE);
    int rp0 = 0, rpn = 0;
    MF_CUDA(cudaMemcpyAsync(&rp0, d_rowptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaMemcpyAsync(&rpn, d_rowptr + rowA, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    const int nnz = rpn - rp0;
    if (nnz < 0) { set_last_error("rowptr[rowA] < rowptr[0]"); return MF_ERR_INVALID_ARG; }

    size_t acc = 0;
    int *d_err = nullptr;
    MF_CUDA(pool_malloc_async(&d_err, sizeof(int) * 8, s));
    MF_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int) * 8, s));
    int *d_class_count = d_err + 1;  // [5]
    int *d_maxnz = d_err + 6;
    if (rowA > 0) {
        k_validate<<<grid_for((long long)rowA + nnz, 256), 256, 0, s>>>(rowA, colA, d_rowptr, d_colidx, d_err);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    int h_err = 0;
    MF_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    if (h_err) {
        cudaFreeAsync(d_err, s);
        set_last_error("CSR input invalid: rowptr not monotone or column outside [0, colA)");
        return MF_ERR_INVALID_ARG;
    }

    // pass 1: per tile-row sort
    int *d_perm = nullptr, *d_cnt = nullptr;
    unsigned long long *d_big = nullptr;
    MF_CUDA(pool_malloc_async(&d_perm, sizeof(int) * (size_t)(nnz + rp0 + 1), s));
    MF_CUDA(pool_malloc_async(&d_cnt, sizeof(int) * (size_t)(tilem + 1), s));
    // global sort space only when some tile-row exceeds the shared-memory cap
    MF_CUDA(pool_malloc_async(&d_big, sizeof(unsigned long long) * (size_t)(nnz + rp0 + 1), s));
    MF_TRY(dalloc(&m->d_tile_ptr, tilem + 1, &acc));
    if (tilem > 0) {
        k_sort_tilerows<<<grid_for(tilem, 1) , BUILD_NT, 0, s>>>(tilem, rowA, d_rowptr, d_colidx, d_perm, d_big, d_cnt);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    MF_CUDA(cudaMemsetAsync(d_cnt + tilem, 0, sizeof(int), s));
    int T = 0;
    MF_TRY(exclusive_scan_i32(d_cnt, m->d_tile_ptr, tilem + 1, s, &T));

    MF_TRY(dalloc(&m->d_tile_columnidx, T, &acc));
    MF_TRY(dalloc(&m->d_tile_nnz, T + 1, &acc));
    MF_TRY(dalloc(&m->d_csrptr_offset, T + 1, &acc));
    MF_TRY(dalloc(&m->d_blknnznnz, T + 1, &acc));
    MF_TRY(dalloc(&m->d_tile_rowidx, T, &acc));
    MF_TRY(dalloc(&m->d_val, nnz, &acc));
    MF_TRY(dalloc(&m->d_val_low, nnz, &acc));
    MF_TRY(dalloc(&m->d_col, nnz, &acc));
    MF_TRY(dalloc(&m->d_cidx, (nnz + 1) / 2, &acc));
    MF_CUDA(cudaMemsetAsync(m->d_cidx, 0, (size_t)(nnz + 1) / 2 + 1, s));
    int *d_run = nullptr;
    MF_CUDA(pool_malloc_async(&d_run, sizeof(int) * (size_t)T * MF_TILE + 16, s));
    MF_CUDA(cudaMemsetAsync(d_run, 0xff, sizeof(int) * (size_t)T * MF_TILE + 16, s));
    if (tilem > 0) {
        k_fill_tilerows<<<grid_for(tilem, 1), BUILD_NT, 0, s>>>(tilem, rowA, rp0, d_rowptr, d_colidx, d_val, d_val_low,
                                                                d_perm, m->d_tile_ptr, m->d_tile_columnidx, m->d_tile_nnz,
                                                                m->d_tile_rowidx, d_run, m->d_val, m->d_val_low, m->d_col);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    const int csrptrlen = (tilem > 0) ? 0 : 0;  // computed below from csrptr_offset[T]
    (void)csrptrlen;
    int *d_nzr = nullptr;
    MF_TRY(dalloc(&d_nzr, T + 1, &acc));
    m->d_nonzero_row_new = d_nzr;
    // Blockcsr_Ptr size: T*16 minus the short last tile-row
    const int rowlen_last = rowA - (tilem - 1) * MF_TILE;
    int last_begin = 0;
    if (tilem > 0) {
        MF_CUDA(cudaMemcpyAsync(&last_begin, m->d_tile_ptr + tilem - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        MF_CUDA(cudaStreamSynchronize(s));
    }
    const int ptrlen = (tilem > 0) ? last_begin * MF_TILE + (T - last_begin) * rowlen_last : 0;
    MF_TRY(dalloc(&m->d_ptr, ptrlen, &acc));
    if (T > 0) {
        k_tile_finish<<<grid_for(T, 256), 256, 0, s>>>(tilem, rowA, T, m->d_tile_ptr, m->d_tile_rowidx, m->d_tile_nnz,
                                                       d_run, m->d_csrptr_offset, m->d_ptr, m->d_blknnznnz, d_nzr, d_err,
                                                       nnz);
        note_launch();
    } else {
        k_tile_finish<<<1, 32, 0, s>>>(tilem, rowA, 0, m->d_tile_ptr, m->d_tile_rowidx, m->d_tile_nnz, d_run,
                                       m->d_csrptr_offset, m->d_ptr, m->d_blknnznnz, d_nzr, d_err, nnz);
        note_launch();
    }
    MF_CUDA(cudaGetLastError());
    MF_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(d_run, s);
    cudaFreeAsync(d_perm, s);
    cudaFreeAsync(d_big, s);
    if (h_err) {
        cudaFreeAsync(d_err, s);
        cudaFreeAsync(d_cnt, s);
        set_last_error("a 16x16 tile holds more than 256 entries (duplicate entries); u8 row pointers cannot describe it");
        return MF_ERR_UNSUPPORTED;
    }

    // non-empty-row lists
    MF_CUDA(cudaMemsetAsync(d_nzr + T, 0, sizeof(int), s));
    int cnt_non = 0;
    MF_TRY(exclusive_scan_i32(d_nzr, d_nzr, T + 1, s, &cnt_non));
    MF_TRY(dalloc(&m->d_blockrowid_new, cnt_non + 1, &acc));
    MF_TRY(dalloc(&m->d_blockcsr_ptr_new, cnt_non + 1, &acc));
    MF_CUDA(cudaMemsetAsync(m->d_blockrowid_new, 0, cnt_non + 1, s));
    MF_CUDA(cudaMemsetAsync(m->d_blockcsr_ptr_new, 0, cnt_non + 1, s));
    if (T > 0) {
        k_nonzero_lists<<<grid_for(T, 256), 256, 0, s>>>(tilem, rowA, T, m->d_tile_rowidx, m->d_tile_nnz,
                                                         m->d_csrptr_offset, m->d_ptr, d_nzr, m->d_blockrowid_new,
                                                         m->d_blockcsr_ptr_new);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }

    // row-block schedule
    MF_TRY(dalloc(&m->d_block_signal, tilem + 1, &acc));
    int rbb = 0;
    {
        int *d_rc = nullptr;
        MF_CUDA(pool_malloc_async(&d_rc, sizeof(int) * (tilem + 1), s));
        k_rbb_count<<<grid_for(tilem + 1, 256), 256, 0, s>>>(tilem, m->d_tile_ptr, d_rc, m->d_block_signal);
        note_launch();
        MF_CUDA(cudaGetLastError());
        MF_TRY(exclusive_scan_i32(d_rc, d_rc, tilem + 1, s, &rbb));
        MF_TRY(dalloc(&m->d_rbb_rowidx, rbb, &acc));
        MF_TRY(dalloc(&m->d_rbb_colstart, rbb, &acc));
        MF_TRY(dalloc(&m->d_rbb_colstop, rbb, &acc));
        if (tilem > 0) {
            k_rbb_fill<<<grid_for(tilem, 256), 256, 0, s>>>(tilem, m->d_tile_ptr, d_rc, m->d_rbb_rowidx,
                                                            m->d_rbb_colstart, m->d_rbb_colstop);
            note_launch();
            MF_CUDA(cudaGetLastError());
        }
        cudaFreeAsync(d_rc, s);
    }

    // payloads and static classes
    MF_TRY(dalloc(&m->d_f16, nnz, &acc));
    MF_TRY(dalloc(&m->d_i8, nnz, &acc));
    MF_TRY(dalloc(&m->d_class, T, &acc));
    MF_TRY(dalloc(&m->d_f16ok, T, &acc));
    if (T > 0) {
        k_payloads<<<grid_for(T, 256), 256, 0, s>>>(T, m->d_tile_nnz, m->d_val, m->d_val_low, m->d_f16, m->d_i8,
                                                    m->d_class, m->d_f16ok, d_class_count, d_maxnz);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    int host_counts[8] = {0};
    MF_CUDA(cudaMemcpyAsync(host_counts, d_err, sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(d_err, s);
    cudaFreeAsync(d_cnt, s);

    m->v.rows = rowA;
    m->v.cols = colA;
    m->v.nnz = nnz;
    m->v.tilem = tilem;
    m->v.tilen = tilen;
    m->v.tilenum = T;
    m->v.csrptrlen = ptrlen;
    m->v.rows_multiple_of_16 = (rowA % MF_TILE) == 0;
    m->v.tile_ptr = m->d_tile_ptr;
    m->v.tile_columnidx = m->d_tile_columnidx;
    m->v.tile_nnz = m->d_tile_nnz;
    m->v.csrptr_offset = m->d_csrptr_offset;
    m->v.val = m->d_val;
    m->v.val_low = m->d_val_low;
    m->v.col = m->d_col;
    m->v.ptr = m->d_ptr;
    m->v.val_f16 = m->d_f16;
    m->v.val_i8 = m->d_i8;
    m->v.tile_class = m->d_class;
    for (int c = 0; c < 5; c++) m->class_tiles[c] = host_counts[1 + c];
    m->max_tile_nnz = host_counts[6];
    m->nonzero_rows = cnt_non;
    m->last_tile_begin = last_begin;
    m->rowblkblock = rbb;
    m->device_bytes = acc;
    return MF_OK;
}

mf_status strip_partition(mf_matrix m, int ctas, cudaStream_t s)
{
    if (m->part_ctas == ctas && m->d_part) return MF_OK;
    if (m->d_part) cudaFree(m->d_part);
    m->d_part = nullptr;
    m->part_ctas = 0;
    const int tilem = m->v.tilem;
    MF_CUDA(cudaMalloc(&m->d_part, sizeof(int) * (ctas + 1)));
    int *d_cost = nullptr;
    MF_CUDA(pool_malloc_async(&d_cost, sizeof(int) * (tilem + 1), s));
    k_strip_cost<<<grid_for(tilem + 1, 256), 256, 0, s>>>(tilem, m->d_tile_ptr, m->d_tile_nnz, d_cost);
    note_launch();
    MF_CUDA(cudaGetLastError());
    MF_TRY(exclusive_scan_i32(d_cost, d_cost, tilem + 1, s, nullptr));
    k_strip_split<<<grid_for(ctas + 1, 256), 256, 0, s>>>(tilem, ctas, d_cost, m->d_part);
    note_launch();
    MF_CUDA(cudaGetLastError());
    cudaFreeAsync(d_cost, s);
    m->part_ctas = ctas;
    return MF_OK;
}

}  // namespace mf
