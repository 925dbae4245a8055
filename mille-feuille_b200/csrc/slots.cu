// slots.cu -- the row-slot execution layout of the persistent solvers.
//
// The tiled format spends its bytes well but costs many instructions per
// row: a row of a strip meets ~7 tiles with ~1 entry each, and every tile
// means pointer and offset loads before its single product.  The solvers
// therefore run from a second, execution-only layout built once per matrix
// from the tiles:
//   * a strip (16 rows) holds K slots, K = the most entries any of its rows
//     has; slot k holds the k-th entry of each of the 16 rows, so one
//     half-warp reads a slot as 16 consecutive elements;
//   * per entry a 16-bit word (tile index within the strip << 4 | in-tile
//     column; 0xFFFF = empty) and the FP64 value; the column is
//     tile_columnidx[tile_ptr[strip] + tile] * 16 + in-tile column;
//   * a row's entries keep the reference's order (tiles in column order,
//     entries in tile order), and the tile index tells where a tile's
//     partial sum ends, so the FP64 row sums round exactly as blockspmv_cpu
//     (src/blockspmv_cpu.h:85-111) does;
//   * mixed precision: every slot stores its 16 values in one format, the
//     widest working class among its entries (fp32 > fp16 > int8 > none).
//     Each value is first rounded to its own tile's working class, and a
//     narrower class is exactly representable in a wider one, so the values
//     the FP32 accumulation sees are those of the per-tile classes; bypassed
//     tiles contribute zeros.  Slot headers: payload offset in 16-byte units
//     << 2 | format (0 fp32, 1 fp16, 2 int8, 3 none).
// Strips with more than 4096 tiles cannot be described by the 16-bit word;
// a matrix with one keeps the chunked tile path.
#include <cuda_fp16.h>

#include <climits>

#include "solver.h"

namespace mf {
namespace {

constexpr int SLOT_MAX_TILES = 4096;

int grid_for3(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

__device__ __forceinline__ void row_bounds(const MfTiles &A, int t, int r, int rowlen, int nz, int &lo, int &hi)
{
    const int po = A.csrptr_offset[t];
    lo = A.ptr[po + r];
    hi = (r == rowlen - 1) ? nz : (int)A.ptr[po + r + 1];
}

// K of every strip (half-warp per strip); flags strips with too many tiles.
__global__ void k_slot_count(MfTiles A, int *__restrict__ K, int *__restrict__ too_many)
{
    const int hl = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s <= A.tilem; s += (gridDim.x * blockDim.x) >> 4) {
        if (s == A.tilem) {
            if (hl == 0) K[s] = 0;
            continue;
        }
        const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
        const int t0 = A.tile_ptr[s], t1 = A.tile_ptr[s + 1];
        int cnt = 0;
        if (hl < rowlen)
            for (int t = t0; t < t1; t++) {
                int lo, hi;
                row_bounds(A, t, hl, rowlen, A.tile_nnz[t + 1] - A.tile_nnz[t], lo, hi);
                cnt += hi - lo;
            }
        for (int o = 8; o > 0; o >>= 1) cnt = max(cnt, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), cnt, o, 16));
        if (hl == 0) {
            K[s] = cnt;
            if (t1 - t0 > SLOT_MAX_TILES) atomicExch(too_many, 1);
        }
    }
}

__global__ void k_slot_fill(MfTiles A, const int *__restrict__ sslot, uint16_t *__restrict__ meta,
                            double *__restrict__ val)
{
    const int hl = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < A.tilem; s += (gridDim.x * blockDim.x) >> 4) {
        const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
        const int t0 = A.tile_ptr[s], t1 = A.tile_ptr[s + 1];
        const size_t base = (size_t)sslot[s] * MF_TILE + hl;
        const int K = sslot[s + 1] - sslot[s];
        int k = 0;
        if (hl < rowlen)
            for (int t = t0; t < t1; t++) {
                const int off = A.tile_nnz[t];
                int lo, hi;
                row_bounds(A, t, hl, rowlen, A.tile_nnz[t + 1] - off, lo, hi);
                for (int q = lo; q < hi; q++, k++) {
                    meta[base + (size_t)k * MF_TILE] = (uint16_t)(((t - t0) << 4) | A.col[off + q]);
                    val[base + (size_t)k * MF_TILE] = A.val[off + q];
                }
            }
        for (; k < K; k++) {
            meta[base + (size_t)k * MF_TILE] = 0xFFFFu;
            val[base + (size_t)k * MF_TILE] = 0.0;
        }
    }
}

// slot format rank of a working class: 0 fp32, 1 fp16, 2 int8, 3 none
__device__ __forceinline__ int class_rank(int c)
{
    return c == MF_CLASS_FP16 ? 1 : c == MF_CLASS_INT8 ? 2 : c == MF_CLASS_BYPASS ? 3 : 0;
}

// Per slot: the widest rank among its entries; size in 16-byte units.
__global__ void k_slot_sizes(MfTiles A, const int *__restrict__ sslot, const uint16_t *__restrict__ meta,
                             const unsigned char *__restrict__ wcls, int nslots, unsigned char *__restrict__ srank,
                             int *__restrict__ sizes)
{
    const int hl = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < A.tilem; s += (gridDim.x * blockDim.x) >> 4) {
        const int t0 = A.tile_ptr[s];
        const int k0 = sslot[s], K = sslot[s + 1] - k0;
        for (int k = 0; k < K; k++) {
            const uint16_t m = meta[((size_t)k0 + k) * MF_TILE + hl];
            int rk = (m == 0xFFFFu) ? 3 : class_rank(wcls[t0 + (m >> 4)]);
            for (int o = 8; o > 0; o >>= 1) rk = min(rk, __shfl_xor_sync(0xFFFFu << (threadIdx.x & 16), rk, o, 16));
            if (hl == 0) {
                srank[k0 + k] = (unsigned char)rk;
                sizes[k0 + k] = rk == 0 ? 4 : rk == 1 ? 2 : rk == 2 ? 1 : 0;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sizes[nslots] = 0;
}

__global__ void k_slot_pack(MfTiles A, const int *__restrict__ sslot, const unsigned char *__restrict__ wcls,
                            const unsigned char *__restrict__ srank, const int *__restrict__ soff,
                            unsigned *__restrict__ shdr, unsigned char *__restrict__ pay)
{
    const int hl = threadIdx.x & 15;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; s < A.tilem; s += (gridDim.x * blockDim.x) >> 4) {
        const int rowlen = (s == A.tilem - 1) ? A.rows - s * MF_TILE : MF_TILE;
        const int t0 = A.tile_ptr[s], t1 = A.tile_ptr[s + 1];
        const int k0 = sslot[s], K = sslot[s + 1] - k0;
        for (int k = hl; k < K; k += MF_TILE) shdr[k0 + k] = ((unsigned)soff[k0 + k] << 2) | srank[k0 + k];
        if (s == A.tilem - 1 && hl == 0) shdr[k0 + K] = ((unsigned)soff[k0 + K] << 2) | 3u;  // end sentinel
        // zero this lane's element of every slot, then write its entries
        for (int k = 0; k < K; k++) {
            unsigned char *d = pay + (size_t)soff[k0 + k] * 16;
            const int rk = srank[k0 + k];
            if (rk == 0) ((float *)d)[hl] = 0.f;
            else if (rk == 1) ((__half *)d)[hl] = __float2half_rn(0.f);
            else if (rk == 2) ((int8_t *)d)[hl] = 0;
        }
        if (hl >= rowlen) continue;
        int k = 0;
        for (int t = t0; t < t1; t++) {
            const int off = A.tile_nnz[t];
            int lo, hi;
            row_bounds(A, t, hl, rowlen, A.tile_nnz[t + 1] - off, lo, hi);
            const int c = wcls[t];
            for (int q = lo; q < hi; q++, k++) {
                const int e = off + q;
                unsigned char *d = pay + (size_t)soff[k0 + k] * 16;
                const int rk = srank[k0 + k];
                // the value in its tile's working class
                float v;
                if (c == MF_CLASS_BYPASS) v = 0.f;
                else if (c == MF_CLASS_FP16) v = __half2float(__ushort_as_half(A.val_f16[e]));
                else if (c == MF_CLASS_INT8) v = (float)A.val_i8[e];
                else v = A.val_low[e];
                // stored in the slot's (equal or wider) format: exact
                if (rk == 0) ((float *)d)[hl] = v;
                else if (rk == 1) ((__half *)d)[hl] = __float2half_rn(v);
                else if (rk == 2) ((int8_t *)d)[hl] = (int8_t)v;
            }
        }
    }
}

constexpr int WALK_NT = 16;  // walking threads per block of the chunk walk kernels

// Sorted union of a staged chunk's tile columns while the walk grows it.
struct StageUnion {
    int n, runs;
    int u[SC_TILES];
    int tmp[SC_TILES];
};

// Merges the (sorted) tile columns tcol[a, b) of one strip into U and counts
// its runs of consecutive tile columns; false, with U unchanged, when the
// union would exceed SC_TILES tile columns or SC_XCAP columns (both only
// grow with the chunk; the run count does not: a strip of a 3D stencil has
// five runs that merge into three once the chunk spans a grid line).
__device__ bool union_add(StageUnion &U, const int *__restrict__ tcol, int a, int b)
{
    int i = 0, j = a, n = 0, runs = 0, prev = -2;
    while (i < U.n || j < b) {
        int v;
        if (j >= b || (i < U.n && U.u[i] <= tcol[j])) {
            v = U.u[i++];
            if (j < b && tcol[j] == v) j++;
        } else {
            v = tcol[j++];
        }
        if (n > 0 && U.tmp[n - 1] == v) continue;
        if (n >= SC_TILES) return false;
        if (v != prev + 1) runs++;
        U.tmp[n++] = v;
        prev = v;
    }
    if (n * MF_TILE > SC_XCAP) return false;
    for (int k = 0; k < n; k++) U.u[k] = U.tmp[k];
    U.n = n;
    U.runs = runs;
    return true;
}

// Greedy chunking of one CTA's strips (the same walk counts and fills): a
// chunk grows while its strips fit the stage and 16 / lanes(max K) half-warp
// groups and, for staged chunks (U given), while its tile columns fit the
// staged vectors; it then ends after the longest prefix whose columns form
// SC_RUNS runs at most, and U is left holding that prefix's union.  A strip
// that cannot be staged on its own becomes a one-strip chunk with staged =
// false.
__device__ int slot_walk(int s, int se, const int *sslot, const int *tile_ptr, const int *tcol, StageUnion *U,
                         bool &direct, int &lanes, bool &staged)
{
    const int s0 = s;
    int kmax = 0, best = -1, best_kmax = 0;
    direct = false;
    staged = U != nullptr;
    if (U) {
        U->n = 0;
        U->runs = 0;
    }
    while (s < se) {
        const int K = sslot[s + 1] - sslot[s];
        const int km = K > kmax ? K : kmax;
        const int nk = sslot[s + 1] - sslot[s0], nt = tile_ptr[s + 1] - tile_ptr[s0];
        if (s - s0 + 1 > SC_STRIPS / slot_lanes(km) || nk > SC_SLOTS || nt > SC_TILES) {
            if (s == s0) {
                direct = true;
                staged = false;
                kmax = km;
                s++;
            }
            break;
        }
        if (U) {
            if (!union_add(*U, tcol, tile_ptr[s], tile_ptr[s + 1])) break;
            if (U->runs <= SC_RUNS) {
                best = s + 1;
                best_kmax = km;
            }
        }
        kmax = km;
        s++;
    }
    if (U && !direct) {
        if (best > s0) {
            s = best;
            kmax = best_kmax;
            // the union of the prefix kept
            U->n = 0;
            U->runs = 0;
            for (int t = s0; t < s; t++) union_add(*U, tcol, tile_ptr[t], tile_ptr[t + 1]);
        } else {
            staged = false;
            s = s0 + 1;
            kmax = sslot[s0 + 1] - sslot[s0];
        }
    }
    lanes = direct ? 16 : slot_lanes(kmax);
    return s;
}

__global__ void k_slot_chunk_count(int G, const int *__restrict__ part, const int *__restrict__ sslot,
                                   const int *__restrict__ tile_ptr, const int *__restrict__ tcol, int staged,
                                   int *__restrict__ cnt)
{
    // the walking thread's tile-column union, in shared memory (WALK_NT
    // threads per block): in local memory its merges went to L2
    __shared__ StageUnion su[WALK_NT];
    StageUnion &U = su[threadIdx.x];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        if (g == G) {
            cnt[g] = 0;
            continue;
        }
        int c = 0, s = part[g];
        const int se = part[g + 1];
        bool d, st;
        int l;
        while (s < se) {
            s = slot_walk(s, se, sslot, tile_ptr, tcol, staged ? &U : nullptr, d, l, st);
            c++;
        }
        cnt[g] = c;
    }
}

__global__ void k_slot_chunk_fill(int G, const int *__restrict__ part, const int *__restrict__ sslot,
                                  const int *__restrict__ tile_ptr, const int *__restrict__ tcol, int staged,
                                  const int *__restrict__ off, SlotChunk *__restrict__ rec, int *__restrict__ unstaged)
{
    // the walking thread's tile-column union, in shared memory (WALK_NT
    // threads per block): in local memory its merges went to L2
    __shared__ StageUnion su[WALK_NT];
    StageUnion &U = su[threadIdx.x];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
        int c = off[g], s = part[g];
        const int se = part[g + 1];
        while (s < se) {
            bool d, st;
            int l;
            const int s1 = slot_walk(s, se, sslot, tile_ptr, tcol, staged ? &U : nullptr, d, l, st);
            SlotChunk r;
            r.s0 = s;
            r.s1 = s1;
            r.k0 = sslot[s];
            r.k1 = sslot[s1];
            r.t0 = tile_ptr[s];
            r.t1 = tile_ptr[s1];
            r.direct = d ? 1 : 0;
            r.lanes = l;
            r.y0 = r.y1 = 0;
            r.fmt = -1;
            r.nrun = -1;
            r.xlen = 0;
            for (int j = 0; j < SC_RUNS; j++) r.rg[j] = r.rl[j] = r.rs[j] = 0;
            if (st) {
                // runs of consecutive tile columns, staged one after another
                int nr = 0, pos = 0;
                for (int k = 0; k < U.n; k++) {
                    if (k == 0 || U.u[k] != U.u[k - 1] + 1) {
                        r.rg[nr] = U.u[k] * MF_TILE;
                        r.rs[nr] = (unsigned short)pos;
                        r.rl[nr] = 0;
                        nr++;
                    }
                    r.rl[nr - 1] = (unsigned short)(r.rl[nr - 1] + MF_TILE);
                    pos += MF_TILE;
                }
                r.nrun = nr;
                r.xlen = pos;
            } else if (staged) {
                atomicAdd(unstaged, 1);
            }
            rec[c++] = r;
            s = s1;
        }
    }
}

// Staged chunks: each slot entry's position in its chunk's staged vectors
// (run start + offset of its column in the run), and each strip's
// descriptor (first slot within the chunk | slots << 16; the offset from a
// row to its own staged position, INT_MIN when the strip's diagonal tile
// column is not staged); one half-warp per strip.
__global__ void k_slot_pos(MfTiles A, int nch, const SlotChunk *__restrict__ rec, const int *__restrict__ sslot,
                           const uint16_t *__restrict__ smeta, uint16_t *__restrict__ spos, int2 *__restrict__ sdesc)
{
    const int hl = threadIdx.x & 15;
    const int nhw = (gridDim.x * blockDim.x) >> 4;
    // half-warp h takes chunk h / 16 and its strips h % 16, h % 16 + 16, ...
    for (long long h = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 4; h < (long long)nch * 16; h += nhw) {
        const SlotChunk &r = rec[h >> 4];
        for (int s = r.s0 + (int)(h & 15); s < r.s1; s += 16) {
            const int t0 = A.tile_ptr[s], k0 = sslot[s], K = sslot[s + 1] - k0;
            if (hl == 0) {
                int od = INT_MIN;
                for (int j = 0; j < r.nrun; j++)
                    if (s * MF_TILE >= r.rg[j] && s * MF_TILE < r.rg[j] + r.rl[j]) od = r.rs[j] - r.rg[j];
                sdesc[s] = make_int2((k0 - r.k0) | (K << 16), od);
            }
            for (int k = 0; k < K; k++) {
                const size_t e = (size_t)(k0 + k) * MF_TILE + hl;
                const uint16_t m = smeta[e];
                uint16_t p = 0xFFFFu;
                if (m != 0xFFFFu && r.nrun >= 0) {
                    const int c0 = A.tile_columnidx[t0 + (m >> 4)] * MF_TILE;
                    for (int j = 0; j < r.nrun; j++)
                        if (c0 >= r.rg[j] && c0 < r.rg[j] + r.rl[j]) p = (uint16_t)(r.rs[j] + (c0 - r.rg[j]) + (m & 15));
                }
                spos[e] = p;
            }
        }
    }
}

// Mixed payload byte range of every chunk (after each packing) and whether
// all its slots share one stored format.
__global__ void k_slot_chunk_pay(int nch, const unsigned *__restrict__ shdr, SlotChunk *__restrict__ rec)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nch; c += gridDim.x * blockDim.x) {
        const int k0 = rec[c].k0, k1 = rec[c].k1;
        rec[c].y0 = (long long)(shdr[k0] >> 2) * 16;
        rec[c].y1 = (long long)(shdr[k1] >> 2) * 16;
        int f = k1 > k0 ? (int)(shdr[k0] & 3u) : -1;
        for (int k = k0 + 1; k < k1 && f >= 0; k++)
            if ((int)(shdr[k] & 3u) != f) f = -1;
        rec[c].fmt = f == 3 ? -1 : f;
    }
}

}  // namespace

mf_status build_slot_chunks(mf_matrix m, int G, bool staged, cudaStream_t s)
{
    const int mode = staged ? 2 : 1;
    if (m->schunk_ctas == G && m->d_schunks && m->schunk_mode == mode) return MF_OK;
    if (m->d_scta_chunk) cudaFree(m->d_scta_chunk);
    if (m->d_schunks) cudaFree(m->d_schunks);
    m->d_scta_chunk = nullptr;
    m->d_schunks = nullptr;
    m->schunk_ctas = 0;
    m->schunk_mode = 0;
    m->schunk_staged = 0;
    MF_CUDA(cudaMalloc(&m->d_scta_chunk, sizeof(int) * (G + 1)));
    int *cnt = nullptr;
    MF_CUDA(pool_malloc_async(&cnt, sizeof(int) * (G + 2), s));
    int *unstaged = cnt + G + 1;
    MF_CUDA(cudaMemsetAsync(unstaged, 0, sizeof(int), s));
    const int *tcol = m->v.tile_columnidx;
    k_slot_chunk_count<<<grid_for3(G + 1, WALK_NT), WALK_NT, 0, s>>>(G, m->d_part, m->d_sslot, m->d_tile_ptr, tcol,
                                                             staged ? 1 : 0, cnt);
    note_launch();
    MF_CUDA(cudaGetLastError());
    int total = 0;
    MF_TRY(exclusive_scan_i32(cnt, m->d_scta_chunk, G + 1, s, &total));
    MF_CUDA(cudaMalloc(&m->d_schunks, sizeof(SlotChunk) * (size_t)(total > 0 ? total : 1)));
    k_slot_chunk_fill<<<grid_for3(G, WALK_NT), WALK_NT, 0, s>>>(G, m->d_part, m->d_sslot, m->d_tile_ptr, tcol,
                                                        staged ? 1 : 0, m->d_scta_chunk, (SlotChunk *)m->d_schunks,
                                                        unstaged);
    note_launch();
    MF_CUDA(cudaGetLastError());
    int h_unstaged = 0;
    MF_CUDA(cudaMemcpyAsync(&h_unstaged, unstaged, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(cnt, s);
    m->nschunks = total;
    m->schunk_ctas = G;
    m->schunk_mode = mode;
    m->schunk_unstaged = h_unstaged;
    if (staged && !h_unstaged) {
        if (!m->d_spos) MF_CUDA(cudaMalloc(&m->d_spos, sizeof(uint16_t) * (size_t)m->nslots * MF_TILE + 32));
        if (!m->d_sdesc) MF_CUDA(cudaMalloc(&m->d_sdesc, sizeof(int2) * ((size_t)m->v.tilem + 2)));
        if (total > 0) {
            k_slot_pos<<<grid_for3((long long)total * 16 * MF_TILE, 256), 256, 0, s>>>(
                m->v, total, (const SlotChunk *)m->d_schunks, m->d_sslot, m->d_smeta, m->d_spos, m->d_sdesc);
            note_launch();
            MF_CUDA(cudaGetLastError());
        }
        m->schunk_staged = 1;
    }
    if (m->d_shdr && m->slot_policy >= 0) {  // payload ranges of an existing packing
        k_slot_chunk_pay<<<grid_for3(total, 256), 256, 0, s>>>(total, m->d_shdr, (SlotChunk *)m->d_schunks);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    return MF_OK;
}

mf_status build_slots(mf_matrix m, cudaStream_t s)
{
    if (m->slots_state != 0) return MF_OK;
    const MfTiles &A = m->v;
    const int tilem = A.tilem;
    int *d_K = nullptr, *d_flag = nullptr;
    MF_CUDA(cudaMalloc(&m->d_sslot, sizeof(int) * (tilem + 1) + 32));  // slack: 16-byte bulk-copy rounding
    MF_CUDA(pool_malloc_async(&d_K, sizeof(int) * (tilem + 1) + sizeof(int), s));
    d_flag = d_K + tilem + 1;
    MF_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
    k_slot_count<<<grid_for3((long long)(tilem + 1) * 16, 256), 256, 0, s>>>(A, d_K, d_flag);
    note_launch();
    MF_CUDA(cudaGetLastError());
    int total = 0, flag = 0;
    MF_TRY(exclusive_scan_i32(d_K, m->d_sslot, tilem + 1, s, &total));
    MF_CUDA(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(d_K, s);
    if (flag || total < 0 || (long long)total * MF_TILE > (1ll << 40)) {
        m->slots_state = -1;  // chunked tile path
        return MF_OK;
    }
    m->nslots = total;
    const size_t E = (size_t)total * MF_TILE;
    MF_CUDA(cudaMalloc(&m->d_smeta, sizeof(uint16_t) * E + 32));
    MF_CUDA(cudaMalloc(&m->d_sval, sizeof(double) * E + 32));
    if (tilem > 0) {
        k_slot_fill<<<grid_for3((long long)tilem * 16, 256), 256, 0, s>>>(A, m->d_sslot, m->d_smeta, m->d_sval);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    m->slots_state = 1;
    m->slot_policy = -1;
    return MF_OK;
}

mf_status pack_slots(mf_matrix m, const unsigned char *d_wcls, cudaStream_t s)
{
    const MfTiles &A = m->v;
    const int ns = (int)m->nslots;
    if (!m->d_shdr) {
        MF_CUDA(cudaMalloc(&m->d_shdr, sizeof(unsigned) * ((size_t)ns + 1) + (size_t)ns + 32));
        MF_CUDA(cudaMalloc(&m->d_spay, (size_t)ns * 64 + 64));
    }
    unsigned char *srank = (unsigned char *)(m->d_shdr + ns + 1);
    int *sizes = nullptr;
    MF_CUDA(pool_malloc_async(&sizes, sizeof(int) * ((size_t)ns + 1) * 2, s));
    int *soff = sizes + ns + 1;
    k_slot_sizes<<<grid_for3((long long)A.tilem * 16, 256), 256, 0, s>>>(A, m->d_sslot, m->d_smeta, d_wcls, ns, srank,
                                                                        sizes);
    note_launch();
    MF_CUDA(cudaGetLastError());
    MF_TRY(exclusive_scan_i32(sizes, soff, ns + 1, s, nullptr));
    if (A.tilem > 0) {
        k_slot_pack<<<grid_for3((long long)A.tilem * 16, 256), 256, 0, s>>>(A, m->d_sslot, d_wcls, srank, soff,
                                                                           m->d_shdr, m->d_spay);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    cudaFreeAsync(sizes, s);
    if (m->d_schunks && m->nschunks > 0) {
        k_slot_chunk_pay<<<grid_for3(m->nschunks, 256), 256, 0, s>>>(m->nschunks, m->d_shdr,
                                                                     (SlotChunk *)m->d_schunks);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    return MF_OK;
}

}  // namespace mf
