// mf_internal.h -- internal (C++) view of the device-resident tiled matrix.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "mf.h"
#include "mf_common.cuh"

// Flat, trivially-copyable view passed to kernels.
struct MfTiles {
    int rows, cols, nnz;
    int tilem, tilen, tilenum, csrptrlen;
    int rows_multiple_of_16;            // 1 when every tile has 16 row pointers
    const int *tile_ptr;                // [tilem+1]
    const int *tile_columnidx;          // [tilenum]
    const int *tile_nnz;                // [tilenum+1] scanned (= blknnz = csr_offset)
    const int *csrptr_offset;           // [tilenum+1]
    const double *val;                  // [nnz] Blockcsr_Val
    const float *val_low;               // [nnz] Blockcsr_Val_Low
    const unsigned char *col;           // [nnz] Tile_csr_Col
    const unsigned char *ptr;           // [csrptrlen] Blockcsr_Ptr
    const uint16_t *val_f16;            // [nnz] fp16 payload bits
    const int8_t *val_i8;               // [nnz] int8 payload
    const unsigned char *tile_class;    // [tilenum] static class
};

struct mf_matrix_s {
    MfTiles v;                 // device pointers (views into the buffers below)
    int device;
    int max_tile_nnz;
    int class_tiles[5];
    int nonzero_rows;          // cnt_non_new
    int last_tile_begin;       // tile_ptr[tilem-1]
    int rowblkblock;
    size_t device_bytes;

    // owned device buffers
    int *d_tile_ptr = nullptr, *d_tile_columnidx = nullptr, *d_tile_nnz = nullptr;
    int *d_csrptr_offset = nullptr;
    unsigned char *d_blknnznnz = nullptr;
    double *d_val = nullptr;
    float *d_val_low = nullptr;
    unsigned char *d_col = nullptr, *d_ptr = nullptr, *d_cidx = nullptr;
    uint16_t *d_f16 = nullptr;
    int8_t *d_i8 = nullptr;
    unsigned char *d_class = nullptr;
    unsigned char *d_f16ok = nullptr;  // per tile: 1 when every FP16 payload value is finite
    // derived reference arrays (src/main-cg.cu:1231-1288, blockspmv_cpu.h:35-83)
    int *d_nonzero_row_new = nullptr, *d_tile_rowidx = nullptr, *d_block_signal = nullptr;
    unsigned char *d_blockrowid_new = nullptr, *d_blockcsr_ptr_new = nullptr;
    unsigned int *d_rbb_rowidx = nullptr;
    int *d_rbb_colstart = nullptr, *d_rbb_colstop = nullptr;
    // strip partitions for the persistent kernels, cached per CTA count
    int part_ctas = 0;
    int *d_part = nullptr;     // [part_ctas+1] strip boundaries
    int *d_cta_chunk = nullptr;  // [part_ctas+1] chunk ranges
    void *d_chunks = nullptr;    // chunk records
    int nchunks = 0;
    // cached per-matrix solver workspace
    void *work = nullptr;
    size_t work_bytes = 0;
    // mixed precision: working class per tile and the packed payload
    unsigned char *d_wcls = nullptr;
    unsigned *d_poff = nullptr;
    unsigned char *d_pay = nullptr;
    size_t pay_bytes = 0, pay_used = 0;
    int packed_policy = -1;
    int policy_loaded = 0;     // a learned policy is attached
    struct mf_policy_s *policy = nullptr;
    void *d_pol = nullptr;     // policy workspace (static tile features, segment statistics)
    size_t pol_bytes = 0;
    int pol_static_ready = 0, pol_have_prev = 0;
    float pol_prev_relres = 0.f;
    // row-slot execution layout of the persistent solvers (slots.cu)
    int slots_state = 0;       // 0 not built, 1 built, -1 not describable
    long long nslots = 0;
    int *d_sslot = nullptr;
    uint16_t *d_smeta = nullptr;
    double *d_sval = nullptr;
    unsigned *d_shdr = nullptr;
    unsigned char *d_spay = nullptr;
    int slot_policy = -1;      // policy whose classes the slot payload holds
    int *d_scta_chunk = nullptr;   // slot chunk table of the current partition
    void *d_schunks = nullptr;
    int schunk_ctas = 0, nschunks = 0;
    int schunk_mode = 0;           // chunks built for: 1 plain, 2 staged
    int schunk_staged = 0;         // 1: staged chunks, every one qualified
    int schunk_unstaged = 0;       // staged build: chunks that did not qualify
    uint16_t *d_spos = nullptr;    // staged positions of the slot entries
    int2 *d_sdesc = nullptr;       // staged strip descriptors
    // per-strip partials of mf_residual_norm
    double *d_resid = nullptr;
    size_t resid_bytes = 0;
    // device staging of b and x for the host-buffer solve entry points
    double *host_io = nullptr;
    size_t host_io_n = 0;
    // multi-right-hand-side solves (multi.cu): interleaved vectors, partials
    // and state, and the staging of the host-array entry point; kept between
    // calls (one solve per matrix at a time, as the buffers above)
    void *mr_work = nullptr;
    size_t mr_work_bytes = 0;
    void *mr_io = nullptr;
    size_t mr_io_bytes = 0;
    // tensor-core SpMM (spmm_tc.cu): dense FP16 copies of the tiles with at
    // least tc_fill entries, and each tile's index among them (-1: sparse)
    int tc_fill = 0;
    int tc_ndense = 0;
    int *d_tc_index = nullptr;
    void *d_tc_dense = nullptr;
};

namespace mf {
// scan.cu
mf_status exclusive_scan_i32(const int *in, int *out, int n, cudaStream_t s, int *total_host);
// tile_build.cu
mf_status build_tiles(mf_matrix m, int rowA, int colA, const int *d_rowptr, const int *d_colidx,
                      const double *d_val, const float *d_val_low, cudaStream_t s);
mf_status strip_partition(mf_matrix m, int ctas, cudaStream_t s);
// spmv.cu
mf_status spmv_fp64(const MfTiles &A, const double *x, double *y, cudaStream_t s);
mf_status spmv_fp64_cidx(const MfTiles &A, const unsigned char *cidx, const double *x, double *y, cudaStream_t s);
// residual.cu: per-strip partials (2 doubles per strip) then a fixed-order sum
mf_status residual_norm(const MfTiles &A, const double *b, const double *x, double *part, double *out,
                        cudaStream_t s);
// workspace
mf_status ensure_work(mf_matrix m, size_t bytes);
}  // namespace mf
