/*
 * ref_wrap.c -- exports the reference's own CPU code for the tiled path as
 * a shared library (oracle/_ref/libmfref.so), so tests can pin the oracle
 * restatement and bench.py can time the reference's CPU path.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference sources are not copied: this file
 * #includes them where they lie (REF_SRC, passed by oracle/Makefile with -I),
 * and only adds flat entry points that copy the reference's results into
 * caller-provided buffers.
 *
 * Wrapped reference functions:
 *   Tile_create      src/csr2block.h:267
 *   encode           src/encode.h:29
 *   blockspmv_cpu    src/blockspmv_cpu.h:2
 *   read_Dmatrix_32  src/biio2.0/src/biio.h:153 (mmio_highlevel.h:7,151)
 */
#include <stdint.h>
#include "csr2block.h"
#include "blockspmv_cpu.h"
#include "biio.h"

typedef struct {
    int tilem, tilen, tilenum, csrsize, csrptrlen;
} ref_tile_sizes;

static Tile_matrix *g_last = NULL;

static void ref_free_matrix(Tile_matrix *m)
{
    if (!m) return;
    free(m->tile_ptr); free(m->tile_columnidx); free(m->tile_nnz); free(m->Format);
    free(m->blknnz); free(m->blknnznnz); free(m->tilewidth); free(m->csr_offset);
    free(m->csrptr_offset); free(m->Blockcsr_Val); free(m->Blockcsr_Val_Low);
    free(m->Blockcsr_Ptr); free(m->csr_compressedIdx); free(m->Tile_csr_Col);
    free(m);
}

/* Runs the reference Tile_create and keeps the result for ref_tile_fetch. */
int ref_tile_create(int rowA, int colA, int nnzA, int *rowptr, int *colidx, double *val,
                    float *val_low, ref_tile_sizes *sz)
{
    ref_free_matrix(g_last);
    g_last = (Tile_matrix *)calloc(1, sizeof(Tile_matrix));
    Tile_create(g_last, rowA, colA, nnzA, rowptr, colidx, val, val_low);
    sz->tilem = g_last->tilem; sz->tilen = g_last->tilen; sz->tilenum = g_last->tilenum;
    sz->csrsize = g_last->csrsize; sz->csrptrlen = g_last->csrptrlen;
    return 0;
}

void ref_tile_fetch(int *tile_ptr, int *tile_columnidx, int *tile_nnz, int *blknnz,
                    unsigned char *blknnznnz, int *csr_offset, int *csrptr_offset,
                    double *vals, float *vals_low, unsigned char *cols, unsigned char *ptr,
                    unsigned char *compressed)
{
    Tile_matrix *m = g_last;
    int T = m->tilenum;
    memcpy(tile_ptr, m->tile_ptr, sizeof(int) * (m->tilem + 1));
    memcpy(tile_columnidx, m->tile_columnidx, sizeof(int) * T);
    memcpy(tile_nnz, m->tile_nnz, sizeof(int) * (T + 1));
    memcpy(blknnz, m->blknnz, sizeof(int) * (T + 1));
    memcpy(blknnznnz, m->blknnznnz, T + 1);
    memcpy(csr_offset, m->csr_offset, sizeof(int) * (T + 1));
    memcpy(csrptr_offset, m->csrptr_offset, sizeof(int) * (T + 1));
    memcpy(vals, m->Blockcsr_Val, sizeof(double) * m->csrsize);
    memcpy(vals_low, m->Blockcsr_Val_Low, sizeof(float) * m->csrsize);
    memcpy(cols, m->Tile_csr_Col, m->csrsize);
    memcpy(ptr, m->Blockcsr_Ptr, m->csrptrlen);
    int cs = m->csrsize % 2 == 0 ? m->csrsize / 2 : m->csrsize / 2 + 1;
    memcpy(compressed, m->csr_compressedIdx, cs);
}

/* Fills csr_compressedIdx with the reference's own encode() over the whole
 * in-tile column array.  The reference allocates this array but never calls
 * encode (its blockspmv_cpu reads it zero-filled); the CPU baseline fills it
 * first so that blockspmv_cpu computes a real product. */
void ref_encode_last(void)
{
    Tile_matrix *m = g_last;
    encode(m->Tile_csr_Col, m->csr_compressedIdx, m->csrsize, 0);
}

void ref_encode(unsigned char *str, unsigned char *res, int str_len, int offset)
{
    encode(str, res, str_len, offset);
}

/* One call of the reference blockspmv_cpu on the last created matrix,
 * including its per-call schedule allocation, as the reference does. */
int ref_blockspmv(int rowA, int colA, int nnzA, double *x, double *y, int *ptroffset1,
                  int *ptroffset2, unsigned int *rowidx_out, int *colstart_out,
                  int *colstop_out)
{
    Tile_matrix *m = g_last;
    int rowblkblock = 0;
    unsigned int *ri; int *cs, *ce;
    blockspmv_cpu(m, ptroffset1, ptroffset2, &rowblkblock, &ri, &cs, &ce, rowA, colA, nnzA,
                  NULL, NULL, NULL, x, y, NULL);
    if (rowidx_out) {
        memcpy(rowidx_out, ri, sizeof(unsigned int) * rowblkblock);
        memcpy(colstart_out, cs, sizeof(int) * rowblkblock);
        memcpy(colstop_out, ce, sizeof(int) * rowblkblock);
    }
    free(ri); free(cs); free(ce);
    return rowblkblock;
}

/* Matrix Market reader: two calls (sizes, then data) around the reference
 * read_Dmatrix_32. */
static int g_m, g_n, g_nnz;
static int *g_rp, *g_ci; static double *g_v;

int ref_read_mtx(char *path, int *m, int *n, int *nnz)
{
    int sym = 0;
    free(g_rp); free(g_ci); free(g_v); g_rp = NULL; g_ci = NULL; g_v = NULL;
    read_Dmatrix_32(&g_m, &g_n, &g_nnz, &g_rp, &g_ci, &g_v, &sym, path);
    *m = g_m; *n = g_n; *nnz = g_nnz;
    return sym;
}

void ref_read_mtx_fetch(int *rp, int *ci, double *v)
{
    memcpy(rp, g_rp, sizeof(int) * (g_m + 1));
    memcpy(ci, g_ci, sizeof(int) * g_nnz);
    memcpy(v, g_v, sizeof(double) * g_nnz);
}

/* CPU baseline: `iters` iterations of FP64 CG whose SpMV is one call of the
 * reference blockspmv_cpu per iteration (its schedule allocation included,
 * as the reference does per call), on the last created (and encoded)
 * matrix.  The reference has no CPU CG; the vector updates and dot products
 * are this harness's own loops, OpenMP-parallel over `threads` threads.
 * Returns the elapsed wall time in seconds; x, r, p are caller buffers of
 * tilen*16 doubles (x0 = 0, r = p = b on entry when start != 0). */
double ref_cg_iterations(int rowA, int colA, int nnzA, const double *b, double *x, double *r, double *p,
                         double *q, int iters, int threads, int start, double *rho_io)
{
    Tile_matrix *m = g_last;
    int n = rowA;
    int *p1 = (int *)malloc(sizeof(int) * (m->tilenum + 1));
    int *p2 = (int *)malloc(sizeof(int) * (m->tilenum + 1));
    omp_set_num_threads(threads);
    double rho = *rho_io;
    if (start) {
        rho = 0;
#pragma omp parallel for reduction(+ : rho)
        for (int i = 0; i < n; i++) { x[i] = 0; r[i] = b[i]; p[i] = b[i]; rho += b[i] * b[i]; }
    }
    double t0 = omp_get_wtime();
    for (int it = 0; it < iters; it++) {
        int rbb; unsigned int *ri; int *cs, *ce;
        blockspmv_cpu(m, p1, p2, &rbb, &ri, &cs, &ce, rowA, colA, nnzA, NULL, NULL, NULL, p, q, NULL);
        free(ri); free(cs); free(ce);
        double pq = 0;
#pragma omp parallel for reduction(+ : pq)
        for (int i = 0; i < n; i++) pq += p[i] * q[i];
        double alpha = rho / pq, rr = 0;
#pragma omp parallel for reduction(+ : rr)
        for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; rr += r[i] * r[i]; }
        double beta = rr / rho;
        rho = rr;
#pragma omp parallel for
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
    }
    double t1 = omp_get_wtime();
    *rho_io = rho;
    free(p1); free(p2);
    return t1 - t0;
}
