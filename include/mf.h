/*
 * mf.h -- C ABI of libmf, the B200 (sm_100a) implementation of the
 * Mille-feuille tiled sparse solver path.
 *
 * Plain C types only.  Device pointers are CUDA global-memory addresses on
 * the current device; `stream` is a cudaStream_t passed as void* (NULL =
 * the legacy default stream).  Every call returns an mf_status; a failing
 * call leaves a message for mf_last_error().  No call aborts the process.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   mf_matrix_create        Tile_create              src/csr2block.h:267
 *                           + host preprocessing      src/main-cg.cu:1231-1454
 *   mf_matrix_destroy       Tile_destroy             src/format.h:88
 *   mf_matrix_export        the Tile_matrix fields   src/format.h:14-86
 *   mf_encode_column_index  encode                   src/encode.h:29
 *   mf_spmv                 stir_spmv_cuda_kernel_newcsr  src/Mille-feuille-cg.h:97
 *                           / blockspmv_cpu          src/blockspmv_cpu.h:2
 *   mf_cg_solve             persistent CG kernels    src/Mille-feuille-cg.h:168,352,1109
 *                           mixed persistent CG      src/main-cg-mixed.cu:99,998
 *   mf_read_matrix_market   read_Dmatrix_32 (.mtx)   src/biio2.0/src/biio.h:153
 *   mf_read_matrix          read_Dmatrix_32          src/biio2.0/src/biio.h:153
 *   mf_matrix_create_mtx    read_Dmatrix_32 +        src/biio2.0/src/biio.h:153,
 *                           Tile_create              src/csr2block.h:267
 *   mf_read_cbd / _write_cbd binary_read_csr /       src/biio2.0/src/biio.h:22, 72
 *                           binary_write_csr
 * The reference's own solve entry points (cg_solve_*, bicgstab*) keep their
 * signatures in Mille-feuille-cg.h / Mille-feuille-bicg.h beside this file.
 */
#ifndef MF_H
#define MF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mf_status {
    MF_OK = 0,
    MF_ERR_INVALID_ARG = 1,  /* bad size, null pointer, index out of range */
    MF_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    MF_ERR_NO_MEMORY = 3,    /* device or host allocation failed */
    MF_ERR_TIMEOUT = 4,      /* a bounded grid-wide wait expired inside a kernel */
    MF_ERR_BREAKDOWN = 5,    /* solver breakdown (zero or non-finite denominator) */
    MF_ERR_NOT_CONVERGED = 6,/* maxiter reached before the tolerance */
    MF_ERR_IO = 7,           /* file could not be read or parsed */
    MF_ERR_UNSUPPORTED = 8,  /* valid input this build does not handle */
    MF_ERR_NO_DEVICE = 9     /* no CUDA device / unsupported architecture */
} mf_status;

/* Text of the last error raised on the calling thread ("" if none). */
const char *mf_last_error(void);
/* Library version string. */
const char *mf_version(void);
/* Kernel launches issued by the library since it was loaded. */
long long mf_kernel_launches(void);

/* ---------------------------------------------------------------------- */
/* Tiled matrix                                                            */
/* ---------------------------------------------------------------------- */

/* Device-resident 16x16 tiled matrix: the reference's tile-CSR arrays,
 * bit-exact, plus the derived schedules and the per-class payloads. */
typedef struct mf_matrix_s *mf_matrix;

/* Static (value-range) precision classes of a tile.  The codes follow the
 * reference's class codes (src/main-cg-mixed.cu:236-322). */
enum {
    MF_CLASS_FP64 = 0,
    MF_CLASS_BYPASS = 1,
    MF_CLASS_INT8 = 2,
    MF_CLASS_FP16 = 3,
    MF_CLASS_FP32 = 4
};

typedef struct mf_matrix_info {
    int rows;           /* rowA: tiled rows */
    int cols;           /* colA */
    int nnz;            /* entries in the first `rows` rows (= csrsize) */
    int tilem, tilen, tilenum, csrsize, csrptrlen;
    int nonzero_rows;   /* cnt_non_new: entries of the non-empty-row lists */
    int rowblkblock;    /* entries of the blockspmv_cpu schedule */
    int class_tiles[5]; /* tiles per static class, indexed by MF_CLASS_* */
    int max_tile_nnz;
    size_t device_bytes;
} mf_matrix_info;

/*
 * Builds the tiled matrix from CSR rows [0, rowA) on the GPU.
 * rowptr has rowA+1 entries (rowptr[0] may be nonzero), column indices must
 * lie in [0, colA).  val_low may be NULL (then (float)val is used).
 * on_device = 0: the four arrays are host memory (copied in), 1: device.
 * Tiles with more than 256 entries (only possible with duplicate entries)
 * are rejected with MF_ERR_UNSUPPORTED: the reference's u8 in-tile row
 * pointers cannot describe them.
 */
mf_status mf_matrix_create(int rowA, int colA, const int *rowptr, const int *colidx,
                           const double *val, const float *val_low, int on_device,
                           void *stream, mf_matrix *out);
mf_status mf_matrix_destroy(mf_matrix m);
mf_status mf_matrix_get_info(mf_matrix m, mf_matrix_info *info);

/*
 * Copies one array of the tiled matrix to host memory.  Names (and element
 * types) follow the reference: tile_ptr, tile_columnidx, tile_nnz, blknnz,
 * csr_offset, csrptr_offset, ptroffset1, ptroffset2 (int32); blknnznnz,
 * Tile_csr_Col, Blockcsr_Ptr, csr_compressedIdx, blockrowid_new,
 * blockcsr_ptr_new (u8); Blockcsr_Val (f64); Blockcsr_Val_Low (f32);
 * nonzero_row_new, tile_rowidx, block_signal (int32); rowblkblock_rowidx
 * (u32), rowblkblock_colstart, rowblkblock_colstop (int32);
 * tile_class (u8, MF_CLASS_*); tile_f16ok (u8: bit 0 every FP16 payload
 * value of the tile is finite, bit 1 every nonzero one is also a normal
 * binary16 number); payload_f16 (u16 bits); payload_i8 (i8).
 * `bytes` must equal the array's size; mf_matrix_array_bytes tells it.
 */
mf_status mf_matrix_array_bytes(mf_matrix m, const char *name, size_t *bytes);
mf_status mf_matrix_export(mf_matrix m, const char *name, void *host_dst, size_t bytes);

/* Packs the in-tile column indices two per byte into csr_compressedIdx,
 * as the reference's encode() over the whole array (src/encode.h:29). */
mf_status mf_encode_column_index(mf_matrix m, void *stream);

/* ---------------------------------------------------------------------- */
/* SpMV and solvers                                                        */
/* ---------------------------------------------------------------------- */

/* y = A x in FP64 (device pointers; x has tilen*16 entries readable, y has
 * rows entries).  Row sums follow blockspmv_cpu's order: per tile a
 * sequential sum over the row's entries, tiles added in column order. */
mf_status mf_spmv(mf_matrix m, const double *x, double *y, void *stream);

/* FP64 true relative residual ||b - A x|| / ||b|| of a square system (the
 * reference's post-solve check, src/main-cg.cu:978-1011): out (device) gets
 * out[0] = relative residual, out[1] = ||b - A x||, out[2] = ||b||.  Rows of
 * A x in blockspmv_cpu's order; per-strip partials summed in a fixed order,
 * so the value is identical on every call.  Scratch: 16 bytes per 16-row
 * strip, allocated on the handle at the first call. */
mf_status mf_residual_norm(mf_matrix m, const double *b, const double *x, double *out, void *stream);

/* Same result as mf_residual_norm, for callers that may not allocate device
 * memory on this path (device memory sized once at start-up, memory owned by
 * the caller's own allocator, or no tolerance for the device-wide
 * synchronisation cudaMalloc/cudaFree can cause).  No counterpart in the
 * reference.  It allocates nothing: its scratch is a fixed 1 MiB array in the
 * library's device image, so it accepts matrices of at most 1,048,576 rows
 * (65,536 strips) and rejects larger ones with MF_ERR_INVALID_ARG.  The first
 * call on a device looks up that array's device address (once per device);
 * make that first call before any stream capture.  All calls on a device
 * share the array: calls that overlap on the GPU race and must be ordered by
 * the caller. */
mf_status mf_residual_norm_noalloc(mf_matrix m, const double *b, const double *x, double *out, void *stream);

typedef enum mf_policy {
    MF_POLICY_FP64 = 0,    /* plain FP64 tiles and vectors */
    MF_POLICY_STATIC = 1,  /* value-range tile classes, FP32 accumulate,
                              FP64 reliable-update refinement */
    MF_POLICY_RULE = 2,    /* STATIC + the reference's partial-convergence
                              rule per segment (absolute thresholds on
                              |p_new - p_old|, src/main-cg-mixed.cu:415-460) */
    MF_POLICY_LEARNED = 3, /* STATIC + the learned per-tile policy */
    MF_POLICY_RULE_SCALED = 4, /* the rule's thresholds on the change relative
                              to max |p| (no reference counterpart: does not
                              depend on the scale of b) */
    MF_POLICY_STATIC_FP16 = 5 /* STATIC, plus every inexact tile whose nonzero
                              values all lie in binary16's normal range
                              [2^-14, 65504] runs from its FP16 payload (the
                              rounding, <= 2^-11 relative, is corrected by the
                              FP64 reliable updates); CG and BiCGSTAB */
} mf_policy;

typedef struct mf_solve_opts {
    int maxiter;          /* iteration cap */
    double tol;           /* stop when ||r||/||b|| <= tol; tol < 0 runs
                             exactly maxiter iterations (the reference's
                             fixed-count behaviour) */
    int policy;           /* mf_policy */
    double refine_delta;  /* reliable update when ||r|| fell by this factor
                             since the last FP64 residual (mixed policies) */
    double wait_budget_s; /* bound on every grid-wide wait inside a kernel */
    int record_history;   /* keep ||r_k||/||b|| per iteration (see report) */
    int phase_times;      /* fill mf_solve_report.phase_us (device timers) */
    int precond;          /* CG only: 0 none (the reference's method), 1 Jacobi
                             (z = D^-1 r with D the diagonal of A; a zero
                             diagonal entry leaves its row unscaled).  No
                             reference counterpart: the preconditioned
                             method cuts iterations on rows of very different
                             scales.  BiCGSTAB and the batched solver reject
                             it with MF_ERR_UNSUPPORTED. */
} mf_solve_opts;

typedef struct mf_solve_report {
    int iterations;        /* Krylov iterations taken */
    int status;            /* mf_status of the solve */
    int refinements;       /* FP64 true-residual recomputations */
    double relres;         /* recurrence residual ||r||/||b|| at exit */
    double relres_true;    /* FP64 ||b - A x|| / ||b|| recomputed at exit */
    double kernel_ms;      /* device time of the solve kernels */
    long long bytes_moved; /* algorithmic bytes of the solve */
    int grid_ctas;         /* CTAs of the persistent launch */
    /* with opts.phase_times: mean over CTAs of the time (us, whole solve)
     * spent in [0] the SpMV phase, [1] its reduction wait, [2] the vector
     * update phase, [3] its reduction wait, [4] reliable updates, [5] the
     * largest per-CTA SpMV-phase time; inside the SpMV phase: [6] waiting
     * for staged chunks, then for tile chunks [7] building x segments and
     * [8] computing rows, for row slots [7] computing rows and [8] the
     * closing barrier and refill */
    double phase_us[9];
    int layout;            /* execution layout of the solve: 0 tile chunks,
                              1 row slots, 2 staged row slots (the chunk's
                              vector entries copied to shared memory) */
    int fallback_iteration;/* RULE / RULE_SCALED CG: the iteration
                              at which the static classes took over because
                              a refinement cycle under the policy's classes
                              did not halve the FP64 residual; 0 if never */
} mf_solve_report;

/* The classes a rule policy gives every tile for the FP32 direction vectors
 * p_new and p_old (device arrays of cols entries; p_old is the direction of
 * the previous iteration).  It replaces the reference's in-kernel decision
 * (src/main-cg-mixed.cu:415-460, d_vis): MF_POLICY_RULE takes, per 16-row
 * segment s of p, v = max |p_new - p_old| over the segment in FP64 and
 * decides MF_CLASS_FP64 (v > 1e-5), FP32 (1e-6 < v <= 1e-5), FP16
 * (1e-7 < v <= 1e-6), INT8 (1e-8 < v <= 1e-7) or BYPASS; a tile takes the
 * decision of its column segment.  The reference's lanes race on the
 * segment's word; the most precise demand wins here.  MF_POLICY_RULE_SCALED
 * applies the thresholds 1e-6 / 1e-7 / 1e-8 to v / max |p_new| in FP32.
 * decision (device, tilenum bytes, may be NULL) receives the decisions,
 * working (device, tilenum bytes, may be NULL) the class the mixed solver
 * runs each tile in: FP32 for FP64 and FP32 decisions, FP16 for FP16 and for
 * INT8 decisions on non-integer tiles, a narrower exact (value-range) class
 * kept.  BYPASS drops the tile only under MF_POLICY_RULE_SCALED; under the
 * absolute thresholds every segment is BYPASS once |p| falls below 1e-8, so
 * there BYPASS runs like INT8.  Any other policy is MF_ERR_INVALID_ARG. */
mf_status mf_rule_classes(mf_matrix m, int policy, const float *p_new, const float *p_old, unsigned char *decision,
                          unsigned char *working, void *stream);

/* Fills opts with the defaults (maxiter 20000, tol 1e-10, FP64 policy). */
void mf_solve_opts_default(mf_solve_opts *opts);

/* Solves A x = b with one persistent cooperative CG kernel (device
 * pointers, x0 = 0).  `history` (may be NULL) receives maxiter+1 doubles
 * when opts->record_history is set. */
mf_status mf_cg_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts *opts,
                      mf_solve_report *report, double *history, void *stream);

/* Same, with b and x in host memory: copies in, solves, copies out. */
mf_status mf_cg_solve_host(mf_matrix m, const double *b_host, double *x_host,
                           const mf_solve_opts *opts, mf_solve_report *report);

/* Solves A x = b (A need not be symmetric) with one persistent cooperative
 * BiCGSTAB kernel, x0 = 0, shadow residual r0 = b; the algorithm of
 * src/Mille-feuille-bicg.h:202-474, stopped on ||r|| <= tol ||b||.  The
 * mixed policies use the value-range tile classes with FP64 reliable
 * updates (no checkpoint policies for BiCGSTAB). */
mf_status mf_bicgstab_solve(mf_matrix m, const double *b, double *x, const mf_solve_opts *opts,
                            mf_solve_report *report, double *history, void *stream);
mf_status mf_bicgstab_solve_host(mf_matrix m, const double *b_host, double *x_host,
                                 const mf_solve_opts *opts, mf_solve_report *report);

/* ---------------------------------------------------------------------- */
/* Several right-hand sides at once (no reference counterpart)             */
/* ---------------------------------------------------------------------- */

/* Y = A X for k columns (1 <= k <= 16) in FP64, one pass over the matrix for
 * all of them.  X (cols x k) and Y (rows x k) are device arrays, column-major
 * with leading dimensions ldx >= cols and ldy >= rows.  Column j of Y equals
 * mf_spmv of column j of X bit for bit (the same blockspmv_cpu summation
 * order).  k outside 1..16 or a short leading dimension is
 * MF_ERR_INVALID_ARG. */
mf_status mf_spmm(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, void *stream);

/* Y = A X as mf_spmm, with the dense tiles on the tensor cores: every tile
 * with at least dense_fill entries (<= 0: 64; at most 256) whose FP16
 * payload is finite is kept as a dense FP16 block (built on the first call
 * and kept on the handle) and multiplied by warp-level MMA (m16n8k16, FP16
 * inputs, FP32 accumulation); the other tiles use their FP32 values.  X is
 * scaled per column by a power of two and rounded to FP16; Y is written in
 * FP64.  Accuracy: FP16 rounding of the dense tiles and of X (2^-11
 * relative each) with FP32 sums -- the form for mixed-precision multi-RHS
 * work, not a replacement for the exact mf_spmm.  dense_tiles (may be NULL)
 * receives the number of dense tiles.  No reference counterpart (it runs
 * one SpMV per vector). */
mf_status mf_spmm_f16(mf_matrix m, int k, const double *X, int ldx, double *Y, int ldy, int dense_fill,
                      int *dense_tiles, void *stream);

/* Solves A X = B for k right-hand sides (1 <= k <= 16) with k independent
 * FP64 CG recurrences that share every SpMM (the matrix is read once per
 * iteration for all columns).  B and X are device arrays, column-major,
 * ldb / ldx >= rows; X is overwritten (the solve starts from x = 0).
 * opts: tol (per column, relative to ||b_j||; negative runs exactly maxiter
 * iterations), maxiter; the FP64 policy only (others MF_ERR_UNSUPPORTED),
 * no preconditioner.  reports (k entries): per column iterations, status,
 * relres (recurrence) and relres_true (FP64 ||b_j - A x_j|| / ||b_j||);
 * kernel_ms and bytes_moved are those of the whole solve.  Returns MF_OK
 * when every column converged, else the first failing column's status
 * (MF_ERR_NOT_CONVERGED, MF_ERR_BREAKDOWN); the other columns still hold
 * their solutions.  The workspace (5 x rows x 16 doubles at most, and for
 * the host entry point 2 x rows x k for the staging) stays allocated in the
 * matrix handle until mf_matrix_destroy; like the other solves on one
 * handle, calls on the same matrix must not run concurrently. */
mf_status mf_cg_solve_multi(mf_matrix m, int k, const double *B, int ldb, double *X, int ldx,
                            const mf_solve_opts *opts, mf_solve_report *reports, void *stream);
/* The same with host arrays (column-major, leading dimension rows). */
mf_status mf_cg_solve_multi_host(mf_matrix m, int k, const double *B_host, double *X_host,
                                 const mf_solve_opts *opts, mf_solve_report *reports);

/* ---------------------------------------------------------------------- */
/* Learned precision policy                                                */
/* ---------------------------------------------------------------------- */

/* A small MLP (16 tile features -> 32 -> 32 -> 4 classes int8-or-bypass /
 * fp16 / fp32 / fp64; BF16 weights, FP32 accumulation) that picks every
 * tile's class at each checkpoint of a MF_POLICY_LEARNED CG solve.  No
 * reference counterpart: it replaces the reference's fixed rule
 * (src/main-cg-mixed.cu:415-460), which stays available as MF_POLICY_RULE. */
typedef struct mf_policy_s *mf_learned;

int mf_policy_param_count(void);
mf_status mf_policy_create(uint64_t seed, mf_learned *out);
mf_status mf_policy_destroy(mf_learned p);
/* Weights as float (BF16 values), layout W1[32][16], b1[32], W2[32][32],
 * b2[32], W3[4][32], b3[4]. */
mf_status mf_policy_get_params(mf_learned p, float *host, int count);
mf_status mf_policy_set_params(mf_learned p, const float *host, int count);
mf_status mf_policy_save(mf_learned p, const char *path);
mf_status mf_policy_load(const char *path, mf_learned *out);
/* Runs a plain FP64 CG solve of m (b on the device) and, every
 * checkpoint_every iterations, adds (features, label) samples of about one
 * tile in sample_stride to the training set (at most max_samples in all). */
mf_status mf_policy_collect(mf_learned p, mf_matrix m, const double *b, int checkpoint_every, int sample_stride,
                            long long max_samples, long long *samples_out);
mf_status mf_policy_label_counts(mf_learned p, long long counts[4]);
/* Adam on the softmax cross-entropy of the collected samples. */
mf_status mf_policy_train(mf_learned p, int epochs, int batch, float lr, uint64_t seed, double *loss_first,
                          double *loss_last);
/* Gradient of the mean loss over n given samples (host X[n][16], Y[n]) at
 * the current weights, without an update (for gradient checks). */
mf_status mf_policy_eval_grad(mf_learned p, const float *X, const int *Y, int n, float *grad, double *loss);
/* MF_POLICY_LEARNED solves of m use p (NULL detaches). */
mf_status mf_matrix_attach_policy(mf_matrix m, mf_learned p);

/* ---------------------------------------------------------------------- */
/* Batched solves                                                          */
/* ---------------------------------------------------------------------- */

/* Many independent square systems of uneven size held on the device.  No
 * reference counterpart (the reference solves one system per launch). */
typedef struct mf_batch_s *mf_batch;

typedef struct mf_batch_report {
    int systems, failed;
    long long iterations_total;
    int iterations_max;
    int refinements_total;
    double relres_true_max;  /* largest FP64 ||b - A x|| / ||b|| over the systems */
    double kernel_ms;        /* device time of the whole batch */
    int lanes_per_row;       /* schedule used: lanes per row in the SpMV */
    int cluster_ctas;        /* schedule used: CTAs per system (thread-block cluster) */
    int status;
    long long bytes_moved;   /* algorithmic bytes of the batch: the chunk passes
                                in their working classes, the vector streams,
                                the FP64 reliable updates */
    double fp16_share;       /* share of the chunk passes run from FP16 values */
} mf_batch_report;

/* count systems; system s has n[s] rows, CSR rowptr[s] (rowptr[s][0] = 0),
 * colidx[s] in [0, n[s]), val[s] (host pointers).  Storage: each system in
 * column panels of 32,768 columns (a 16-bit column offset within the panel
 * per entry, the panel's rows in CSR); values in FP64, FP32 and FP16 scaled
 * per row by a power of two (diagonal kept apart in FP32; the FP16 value and
 * its column packed in one 32-bit word); rows cut into chunks of at most 256
 * rows and 4,096 entries in every panel, each with a precision class. */
mf_status mf_batch_create(int count, const int *n, const int *const *rowptr, const int *const *colidx,
                          const double *const *val, mf_batch *out);
mf_status mf_batch_destroy(mf_batch bt);
/* Total rows / entries, and the first row of each system in the stacked
 * vectors b and x (host array owned by the handle). */
mf_status mf_batch_info(mf_batch bt, long long *rows_total, long long *nnz_total, const long long **row_offsets);
/* CG on every system (b, x: device arrays of rows_total doubles, stacked in
 * system order).  One launch; use_graph != 0 captures the solve (queue reset,
 * the batched kernel, the FP64 residual check) in a CUDA graph, replayed on
 * later calls with the same buffers and options.  Policies: FP64 (FP64
 * values and vectors), and the mixed policies (FP32 vectors and sums, each
 * chunk read in FP32 or FP16, FP64 reliable updates, convergence on the FP64
 * residual) whose classes are chosen inside the kernel: STATIC (FP16 only
 * for chunks exact in FP16), RULE (every iteration, the reference's
 * thresholds on the chunk rows' |p_new - p_old|: above 1e-6 FP32, else
 * FP16), LEARNED (the attached policy at the first iteration and at every
 * reliable update; MF_ERR_UNSUPPORTED without one).  RULE and LEARNED return
 * to the static classes for the rest of a system's solve when a reliable
 * update finds the FP64 residual above half of the previous one.
 * MF_POLICY_RULE_SCALED and the preconditioner are MF_ERR_UNSUPPORTED. */
mf_status mf_batch_cg_solve(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int use_graph,
                            mf_batch_report *report, void *stream);
/* Per-system iterations and FP64 true relative residuals of the last solve. */
mf_status mf_batch_results(mf_batch bt, int *iterations, double *relres_true);
/* Chunks of the batch, chunks exact in FP16 (the STATIC class), chunks whose
 * rows can be held in FP16 at all (row scales within FP32's range). */
mf_status mf_batch_chunk_count(mf_batch bt, int *chunks, int *static_fp16, int *fp16_capable);
/* Copies one array of the batch to host memory: chunk_class (u8 per chunk:
 * 0 FP32, 1 FP16, the classes at the end of the last solve), chunk_static
 * (u8: bit 0 exact in FP16, bit 1 FP16-capable), chunk_features_static
 * (6 floats per chunk: features 0-4 and the chunk's max |a|), chunk_start
 * (int32, count+1: first chunk of each system), chunk_rows (int32: per
 * system its chunks' first rows and the row count), chunk_ends (int32: the
 * same chunks' first entries and the entry count), val16 (FP16 bits), val32, row_scale, diag32 (float), col (u16:
 * the column offset within its panel).  `bytes` must equal the array's size. */
mf_status mf_batch_export(mf_batch bt, const char *name, void *host_dst, size_t bytes);
/* MF_POLICY_LEARNED batched solves use p (NULL detaches). */
mf_status mf_batch_attach_policy(mf_batch bt, mf_learned p);
/* Runs a plain FP64 batched solve of every system (b on the device) and, at
 * iterations 1, 1 + k, 1 + 2k, ... (k = checkpoint_every), adds (chunk
 * features, label) samples of about one chunk in sample_stride to p's
 * training set (at most max_samples in all).  Label 1 (FP16) when the FP16
 * values perturb the chunk's part of A p by at most 2^-6 of it (2-norms over
 * its rows), else 2 (FP32). */
mf_status mf_batch_policy_collect(mf_learned p, mf_batch bt, const double *b, int checkpoint_every,
                                  int sample_stride, long long max_samples, long long *samples_out);
/* The attached policy's class for every chunk, for given device vectors r,
 * p_new, p_old, q (rows_total doubles each, stacked), per-system relative
 * residuals and reliable-update counts (device arrays of `systems` entries):
 * the classifier the LEARNED solve runs at its checkpoints.  classes
 * (device, one byte per chunk); features (device, 16 floats per chunk, may
 * be NULL).  have_prev = 0 takes the history features from the current
 * checkpoint; every call stores them for the next.  Synchronous. */
mf_status mf_batch_policy_classify(mf_batch bt, const double *r, const double *p_new, const double *p_old,
                                   const double *q, const double *relres, const int *refinements, int have_prev,
                                   unsigned char *classes, float *features);
/* Autotuner: times each schedule (lanes per row 4/8/16/32 x cluster size
 * 1/2/4/8/16; one 512-thread CTA per SM) on this batch, keeps the fastest
 * on the handle.  Default schedule: 4 lanes, clusters of 2 CTAs.  Clusters
 * of 16 CTAs exceed the portable cluster size and are enabled explicitly on
 * the kernel. */
mf_status mf_batch_tune(mf_batch bt, const double *b, double *x, const mf_solve_opts *opts, int *lanes_out,
                        int *cluster_out, void *stream);
/* lanes in {4, 8, 16, 32}, cluster in {1, 2, 4, 8, 16}. */
mf_status mf_batch_set_schedule(mf_batch bt, int lanes, int cluster);

/* Diagnostic: runs the persistent kernels' bounded waits (a grid barrier
 * whose second epoch nobody completes, an mbarrier nobody arrives at) on 2
 * CTAs and reports how they ended: results[0] = the device status word
 * (MF_ERR_TIMEOUT expected), then per CTA {first barrier passed (1), second
 * barrier passed (0), mbarrier wait expired with MF_ERR_TIMEOUT (1)}.  7
 * ints.  budget_s in (0, 10].  No reference counterpart. */
mf_status mf_selftest_bounded_waits(double budget_s, int *results);

/* ---------------------------------------------------------------------- */
/* Matrix Market input and synthetic matrices                              */
/* ---------------------------------------------------------------------- */

/* Reads a Matrix Market coordinate file into host CSR arrays allocated
 * with malloc (free with mf_free_host).  Entry order follows the
 * reference reader: rows in file order, the mirrored entry of a symmetric
 * file placed right after its original (mmio_highlevel.h:151-321). */
mf_status mf_read_matrix_market(const char *path, int *m, int *n, int *nnz, int **rowptr,
                                int **colidx, double **val, int *is_symmetric);

/* A Matrix Market file straight to a device-resident matrix: the entries
 * are parsed on the host threads as mf_read_matrix_market parses them, the
 * CSR (the same arrays, bit for bit) is built on the GPU -- the symmetric
 * mirrors expanded in place, a stable radix sort by row -- and handed to
 * the tile build without a host round trip (read_Dmatrix_32 + Tile_create,
 * src/biio2.0/src/biio.h:153, src/csr2block.h:267).  Stream-ordered on
 * `stream`; returns after the matrix is built. */
mf_status mf_matrix_create_mtx(const char *path, void *stream, mf_matrix *out, int *is_symmetric);

/* Binary CSR files (".cbd"), the reference's cache of a parsed matrix
 * (binary_read_csr / binary_write_csr, src/biio2.0/src/biio.h:22-94):
 * int32 rows, int32 cols, int64 nnz, int64 row_ptr[rows+1],
 * int32 col_idx[nnz], double val[nnz], machine byte order.  The reader
 * allocates with malloc (free with mf_free_host) and reports a file whose
 * length, row pointers or column indices do not match its header as
 * MF_ERR_IO; more than 2^31-1 entries is MF_ERR_UNSUPPORTED. */
mf_status mf_read_cbd(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx, double **val);
mf_status mf_write_cbd(const char *path, int m, int n, int nnz, const int *rowptr, const int *colidx,
                       const double *val);

/* The CLIs' reader (read_Dmatrix_32, src/biio2.0/src/biio.h:153): ".cbd"
 * files through mf_read_cbd (*is_symmetric set to 0: the file holds the
 * matrix as stored), ".mtx" files through mf_read_matrix_market; any other
 * name is MF_ERR_IO. */
mf_status mf_read_matrix(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx, double **val,
                         int *is_symmetric);
void mf_free_host(void *p);

/*
 * Seeded synthetic matrices (host CSR, malloc'd; free with mf_free_host).
 * They stand in for the paper's SuiteSparse inputs.  No reference
 * counterpart: the generator is this library's own.  Randomness is the
 * counter-based SplitMix64 stream u(seed, stream, i) in [0, 1).
 */
double mf_rng_u01(uint64_t seed, uint64_t stream, uint64_t i);
double mf_rng_normal(uint64_t seed, uint64_t stream, uint64_t m);
mf_status mf_synth_xstar(uint64_t seed, int n, double *out);
mf_status mf_synth_laplace2d(int nx, int ny, int *n, int *nnz, int **rowptr, int **colidx, double **val);
mf_status mf_synth_poisson3d_scaled(int g, uint64_t seed, int *n, int *nnz, int **rowptr, int **colidx,
                                    double **val);
mf_status mf_synth_convdiff3d(int g, double peclet, double vx, double vy, double vz, int *n, int *nnz,
                              int **rowptr, int **colidx, double **val);
int mf_synth_random_spd_size(uint64_t seed);
mf_status mf_synth_random_spd(int n, uint64_t seed, int *n_out, int *nnz, int **rowptr, int **colidx,
                              double **val);
mf_status mf_synth_aniso3d(int g, uint64_t seed, double log_sigma, double corr_len, double aniso, int *n,
                           int *nnz, int **rowptr, int **colidx, double **val);

#ifdef __cplusplus
}
#endif
#endif /* MF_H */
