/*
 * Mille-feuille-tile.h -- the reference's tiled-format API (Tile_matrix,
 * Tile_create, Tile_destroy, blockspmv_cpu) served by libmf.
 *
 * The struct keeps the reference's field names, types and order
 * (src/format.h:14-86) so that code written against the reference compiles
 * and reads the same fields; one field is appended at the end
 * (mf_handle: the device-resident matrix libmf built).  Only the 16x16
 * CSR-tile fields are filled, exactly as the reference's Tile_create fills
 * them; every other pointer is NULL and every other count 0.
 *
 *   Tile_create    src/csr2block.h:267   built on the GPU, arrays copied to
 *                                        malloc'd host memory, bit-identical
 *                                        to the reference's
 *   Tile_destroy   src/format.h:88       also releases the device matrix
 *   blockspmv_cpu  src/blockspmv_cpu.h:2 schedule arrays built on the GPU;
 *                                        y = A x computed on the GPU in the
 *                                        reference's order, columns read
 *                                        from csr_compressedIdx as the
 *                                        reference does
 *
 * Unlike the reference these report failures: Tile_create leaves tilem =
 * tilen = tilenum = 0 and all pointers NULL, blockspmv_cpu sets
 * *rowblkblock = -1; mf_last_error() has the message.
 */
#ifndef MILLE_FEUILLE_TILE_H
#define MILLE_FEUILLE_TILE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct csrval {
    double csrval_high;
    float csrval_low;
} mixval;

typedef struct {
    int tilem;
    int tilen;
    int tilenum;
    int *tile_ptr;
    int *tile_columnidx;
    int *tile_nnz;
    char *Format;
    int *blknnz;
    unsigned char *blknnznnz;
    int *dnsrowptr;
    int *dnscolptr;
    char *tilewidth;
    int *csr_offset;
    int *csrptr_offset;
    int *coo_offset;
    int *ell_offset;
    int *hyb_offset;
    int *hyb_coocount;
    int *dns_offset;
    int *dnsrow_offset;
    int *dnscol_offset;
    int *new_coocount;
    double *Blockcsr_Val;
    float *Blockcsr_Val_Low;
    unsigned char *Tile_csr_Col;
    mixval *Blockcsr_Val_mix;
    unsigned char *Blockcsr_Ptr;
    unsigned char *csr_compressedIdx;
    int csrsize;
    int csrptrlen;
    double *Blockcoo_Val;
    float *Blockcoo_Val_Low;
    unsigned char *coo_compressed_Idx;
    int coosize;
    double *Blockell_Val;
    float *Blockell_Val_Low;
    unsigned char *ell_compressedIdx;
    int ellsize;
    double *Blockhyb_Val;
    float *Blockhyb_Val_Low;
    unsigned char *hybIdx;
    int hybsize;
    int hybellsize;
    int hybcoosize;
    double *Blockdense_Val;
    float *Blockdense_Val_Low;
    int dnssize;
    double *Blockdenserow_Val;
    float *Blockdenserow_Val_Low;
    char *denserowid;
    int dnsrowsize;
    double *Blockdensecol_Val;
    float *Blockdensecol_Val_Low;
    char *densecolid;
    int dnscolsize;
    int coototal;
    double *deferredcoo_val;
    float *deferredcoo_val_Low;
    int *deferredcoo_colidx;
    int *deferredcoo_ptr;
    int rowblkblock;
    unsigned int *flag_bal_tile_rowidx;
    int *tile_bal_rowidx_colstart;
    int *tile_bal_rowidx_colstop;
    int *flag_tilerow_start;
    int *flag_tilerow_stop;
    int *tile_bal_rowidx_colstart_v2;
    int *tile_bal_rowidx_colstop_v2;
    int *map;
    void *mf_handle; /* libmf: the device matrix (mf_matrix), or NULL */
} Tile_matrix;

void Tile_create(Tile_matrix *matrix, int rowA, int colA, int nnzA, int *csrRowPtrA, int *csrColIdxA,
                 double *csrValA, float *csrValA_Low);
void Tile_destroy(Tile_matrix *matrix);
void blockspmv_cpu(Tile_matrix *matrix, int *ptroffset1, int *ptroffset2, int *rowblkblock,
                   unsigned int **blkcoostylerowidx, int **blkcoostylerowidx_colstart,
                   int **blkcoostylerowidx_colstop, int rowA, int colA, int nnzA, int *csrRowPtrA,
                   int *csrColIdxA, double *csrValA, double *x, double *y, double *y_golden);

#ifdef __cplusplus
}
#endif
#endif
