// chunks.cu -- per-CTA chunk table of the persistent solver: consecutive
// strips grouped so that one chunk's tiles, entries and bytes fit one
// shared-memory stage, computed once per strip partition.
#include "solver.h"

namespace mf {
namespace {

__device__ __forceinline__ int strip_walk(int s, int se, const int *tile_ptr, const int *tile_nnz, int &tiles_out,
                                          int &ent_out, bool &direct)
{
    // returns s1 of the chunk starting at s
    const int s0 = s;
    int tiles = 0, ent = 0;
    direct = false;
    while (s < se && s - s0 < CH_STRIPS) {
        const int nt = tile_ptr[s + 1] - tile_ptr[s];
        const int ne = tile_nnz[tile_ptr[s + 1]] - tile_nnz[tile_ptr[s]];
        if (tiles + nt > CH_TILES || ent + ne > CH_ENTRIES) {
            if (s == s0) {
                direct = true;
                s++;
            }
            break;
        }
        tiles += nt;
        ent += ne;
        s++;
    }
    tiles_out = tiles;
    ent_out = ent;
    return s;
}

__global__ void k_chunk_count(int G, const int *__restrict__ part, const int *__restrict__ tile_ptr,
                              const int *__restrict__ tile_nnz, int *__restrict__ cnt)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        if (g == G) {
            cnt[g] = 0;
            continue;
        }
        int c = 0, s = part[g];
        const int se = part[g + 1];
        while (s < se) {
            int nt, ne;
            bool d;
            s = strip_walk(s, se, tile_ptr, tile_nnz, nt, ne, d);
            c++;
        }
        cnt[g] = c;
    }
}

__global__ void k_chunk_fill(int G, const int *__restrict__ part, const int *__restrict__ tile_ptr,
                             const int *__restrict__ tile_nnz, const int *__restrict__ off, ChunkRec *__restrict__ rec)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
        int c = off[g], s = part[g];
        const int se = part[g + 1];
        while (s < se) {
            int nt, ne;
            bool d;
            const int s1 = strip_walk(s, se, tile_ptr, tile_nnz, nt, ne, d);
            ChunkRec r;
            r.s0 = s;
            r.s1 = s1;
            r.t0 = tile_ptr[s];
            r.t1 = tile_ptr[s1];
            r.e0 = tile_nnz[r.t0];
            r.e1 = tile_nnz[r.t1];
            r.y0 = 0;
            r.y1 = 0;
            r.direct = d ? 1 : 0;
            r.pad = 0;
            rec[c++] = r;
            s = s1;
        }
    }
}

__global__ void k_chunk_pay(int n, const unsigned *__restrict__ poff, ChunkRec *__restrict__ rec)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        rec[c].y0 = poff[rec[c].t0];
        rec[c].y1 = poff[rec[c].t1];
    }
}

int grid_for3(long long work, int nt)
{
    long long g = (work + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

mf_status build_chunks(mf_matrix m, cudaStream_t s)
{
    const int G = m->part_ctas;
    if (m->d_cta_chunk) cudaFree(m->d_cta_chunk);
    if (m->d_chunks) cudaFree(m->d_chunks);
    m->d_cta_chunk = nullptr;
    m->d_chunks = nullptr;
    MF_CUDA(cudaMalloc(&m->d_cta_chunk, sizeof(int) * (G + 1)));
    k_chunk_count<<<grid_for3(G + 1, 128), 128, 0, s>>>(G, m->d_part, m->d_tile_ptr, m->d_tile_nnz, m->d_cta_chunk);
    note_launch();
    MF_CUDA(cudaGetLastError());
    int total = 0;
    MF_TRY(exclusive_scan_i32(m->d_cta_chunk, m->d_cta_chunk, G + 1, s, &total));
    MF_CUDA(cudaMalloc(&m->d_chunks, sizeof(ChunkRec) * (total > 0 ? total : 1)));
    if (G > 0) {
        k_chunk_fill<<<grid_for3(G, 128), 128, 0, s>>>(G, m->d_part, m->d_tile_ptr, m->d_tile_nnz, m->d_cta_chunk,
                                                       (ChunkRec *)m->d_chunks);
        note_launch();
        MF_CUDA(cudaGetLastError());
    }
    m->nchunks = total;
    return MF_OK;
}

mf_status refresh_chunk_payload(mf_matrix m, cudaStream_t s)
{
    if (m->nchunks == 0 || !m->d_poff) return MF_OK;
    k_chunk_pay<<<grid_for3(m->nchunks, 256), 256, 0, s>>>(m->nchunks, m->d_poff, (ChunkRec *)m->d_chunks);
    note_launch();
    MF_CUDA(cudaGetLastError());
    return MF_OK;
}

}  // namespace mf
