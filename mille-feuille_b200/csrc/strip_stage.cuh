// strip_stage.cuh -- half-warp staging of one 16-row strip (tile-row) into
// shared memory, and the per-row products computed from it.
//
// A strip's tiles are consecutive in every canonical array, so its payload,
// in-tile column bytes and u8 row pointers are three contiguous byte ranges.
// The 16 lanes of a half-warp copy them with 16-byte cp.async (all copies in
// flight at once), load the tile metadata one tile per lane, and build the
// 16-element x segment of every tile of the strip in shared memory with
// coalesced loads.  Lane r then walks the strip's tiles for row r in column
// order, each tile's entries in order -- the summation order of the
// reference's blockspmv_cpu (src/blockspmv_cpu.h:98-108).
#pragma once
#include <cuda_fp16.h>

#include "mf_internal.h"

namespace mf {

constexpr int STAGE_MAXT = 8;     // tiles per strip on the staged path
constexpr int STAGE_CAPE = 128;   // entries per strip on the staged path

// Shared-memory staging area of one half-warp.
struct alignas(16) StripBuf {
    double seg[STAGE_MAXT][MF_TILE];              // x segment of each tile
    unsigned char pay[STAGE_CAPE * 8 + 32];       // payload bytes
    unsigned char col[STAGE_CAPE + 32];           // in-tile column bytes
    unsigned char ptr[STAGE_MAXT * MF_TILE + 32]; // u8 row pointers
    int pshift;                                   // ptr[] offset of tile 0
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Copies bytes [a0, a1) of `src` (16-byte aligned base, 16 bytes of slack
// past the end) into `dst`; returns the aligned start so that byte a lives at
// dst[a - base].  hl = lane within the half-warp.
__device__ __forceinline__ long long stage_range(unsigned char *dst, const unsigned char *src, long long a0,
                                                 long long a1, int hl)
{
    const long long c0 = a0 & ~15ll, c1 = (a1 + 15) & ~15ll;
    for (long long c = c0 + 16ll * hl; c < c1; c += 256) cp_async16(dst + (c - c0), src + c);
    return c0;
}

// Strip descriptor shared by the lanes of a half-warp (held in registers:
// lane j < cnt holds tile j's values).
struct StripMeta {
    int t0, cnt;        // first tile, number of tiles
    int e0;             // first canonical entry of the strip
    int my_tc;          // lane j: tile column of tile j
    int my_off;         // lane j: tile j's first entry, relative to e0
    int my_nz;          // lane j: entries of tile j
    int my_pb;          // lane j: byte offset of tile j's payload in the staged buffer
    int my_cls;         // lane j: payload class of tile j
    bool staged;
};

}  // namespace mf
