/*
 * mf_oracle.h -- CPU oracle for the Mille-feuille solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links this code;
 * it is loaded by tests/, by __graft_entry__.smoke() and by the CPU-baseline
 * leg of bench.py, and only as the checker.
 *
 * Every function restates one piece of the reference algorithm in plain C
 * and cites the reference file:line it follows (paths relative to the
 * reference project root).  The restatement is pinned against the
 * reference's own CPU code, compiled from the reference sources into
 * oracle/_ref/ by oracle/Makefile (see tests/test_oracle_vs_reference.py),
 * and against the committed fixtures in tests/golden/.
 */
#ifndef MF_ORACLE_H
#define MF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Canonical 16x16 tiled CSR format (src/format.h:14-86, CSR fields only). */
typedef struct {
    int tilem, tilen, tilenum, csrsize, csrptrlen;
    int *tile_ptr;            /* [tilem+1]  */
    int *tile_columnidx;      /* [tilenum]  */
    int *tile_nnz;            /* [tilenum+1] exclusive scan */
    int *blknnz;              /* [tilenum+1] exclusive scan */
    unsigned char *blknnznnz; /* [tilenum+1] unscanned counts truncated to u8 */
    int *csr_offset;          /* [tilenum+1] */
    int *csrptr_offset;       /* [tilenum+1] */
    double *Blockcsr_Val;     /* [csrsize] */
    float *Blockcsr_Val_Low;  /* [csrsize] */
    unsigned char *Tile_csr_Col; /* [csrsize] */
    unsigned char *Blockcsr_Ptr; /* [csrptrlen] */
} orc_tiles;

int  orc_tile_create(int rowA, int colA, const int *rowptr, const int *colidx,
                     const double *val, const float *val_low, orc_tiles *out);
void orc_tiles_free(orc_tiles *t);

/* 4-bit index packing (src/encode.h:29-72). */
void orc_encode(const unsigned char *str, unsigned char *res, int str_len, int offset);
void orc_decode(const unsigned char *str, unsigned char *res, int res_len);

/* blockspmv_cpu schedule + SpMV (src/blockspmv_cpu.h:2-112). */
int  orc_rowblkblock_count(const orc_tiles *t);
void orc_blockspmv(const orc_tiles *t, int rowA, int colA, const unsigned char *compressed_idx,
                   int *ptroffset1, int *ptroffset2, unsigned int *rowidx, int *colstart,
                   int *colstop, const double *x, double *y);

/* Non-empty-row compaction (src/main-cg.cu:1231-1288). */
int  orc_nonzero_rows_count(const orc_tiles *t, int rowA);
void orc_nonzero_rows(const orc_tiles *t, int rowA, int *nonzero_row_new, int *tile_rowidx,
                      unsigned char *blockrowid_new, unsigned char *blockcsr_ptr_new,
                      int *block_signal);

/* nnz load balancer of cg_solve_inc (src/main-cg.cu:1290-1454). */
int  orc_balance(const orc_tiles *t, int nnzR, int *index_out, int *each_block_nnz_out,
                 int *balance_tile_ptr, int *row_each_block, int *index_each_block,
                 int *vector_each_warp_32, int *vector_total_32);

/* Low-precision payload casts (src/main-cg-mixed.cu:2325-2342). */
uint16_t orc_f32_to_f16_bits(float f);
float    orc_f16_bits_to_f32(uint16_t h);
void     orc_payload_casts(const double *v, int n, float *f32, uint16_t *f16, int8_t *i8);

/* Per-segment precision rule, race-free restatement of
 * src/main-cg-mixed.cu:415-460. */
int  orc_rule_class(double max_abs_dp);
/* The batched configuration's random SPD generator (see .c); returns n. */
int  orc_random_spd_size(uint64_t seed);
int  orc_random_spd(uint64_t seed, int n, int *nnz_out, int **rowptr, int **colidx, double **val);
void orc_xstar(uint64_t seed, int n, double *out);
void orc_free(void *p);
/* Batched solver storage and chunk policy (see .c). */
uint16_t orc_f64_to_f16_bits(double v);
void orc_batch_rows(int n, const int *rp, const int *ci, const double *val, uint16_t *val16, float *rscale,
                    float *diag32, unsigned char *flag, float *rowstat);
void orc_pn_forward(const float *w, const float *x, float *out);
void orc_batch_classify(int n, const int *rp, const int *ci, const double *val, int nch, const int *crow,
                        const int *cent, const double *r, const double *pn, const double *po, const double *q,
                        double relres, int refs, int have_prev, float *prev, const float *w, float *feat,
                        unsigned char *cls, double *margin);
/* Per-tile rule decision and working class for FP32 directions (see .c). */
void orc_rule_tiles(int n, int tilen, int T, const int *tile_col, const unsigned char *static_cls,
                    const unsigned char *f16ok, const float *pn, const float *po, int scaled, unsigned char *decision,
                    unsigned char *working);

/* CSR SpMV and FP64 solvers (textbook order; sequential sums). */
void orc_csr_spmv(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *x, double *y);
int  orc_cg(int n, const int *rowptr, const int *colidx, const double *val, const double *b,
            double *x, int maxiter, double tol, double *relres_out, double *hist);
int  orc_bicgstab(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *b, double *x, int maxiter, double tol, double *relres_out);
double orc_true_relres(int n, const int *rowptr, const int *colidx, const double *val,
                       const double *b, const double *x);

/* Tiled SpMV with the row-sum order of blockspmv_cpu but reading the
 * uncompressed in-tile column array (the arrays the GPU path uses). */
void orc_tiled_spmv(const orc_tiles *t, int rowA, const double *x, double *y);

/* MLP policy (16 -> 32 -> 32 -> 4): mean softmax cross-entropy over n
 * samples and its gradient, double precision. */
double orc_mlp_grad(const float *w, const float *X, const int *Y, int n, double *grad);

#ifdef __cplusplus
}
#endif
#endif
