// tile_api.cu -- the reference's tiled-format API (Tile_create, Tile_destroy,
// blockspmv_cpu) on top of the GPU tile build.
//
// Tile_create (src/csr2block.h:267-422) builds the tiles with
// mf_matrix_create and copies every array the reference fills into
// malloc'd host memory; csr_compressedIdx is zero-filled, as the reference
// leaves it (it allocates it but never encodes, src/csr2block.h:387-389).
// blockspmv_cpu (src/blockspmv_cpu.h:2-112) returns the row-block schedule
// and the per-tile offsets built on the GPU and computes y = A x on the GPU
// in the reference's summation order with the in-tile columns taken from the
// struct's csr_compressedIdx, which is what the reference reads.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "Mille-feuille-tile.h"
#include "mf_internal.h"

namespace {

template <typename T>
T *export_array(mf_matrix h, const char *name, size_t count, bool &ok)
{
    T *p = (T *)calloc(count ? count : 1, sizeof(T));
    if (!p) {
        ok = false;
        return nullptr;
    }
    size_t bytes = 0;
    if (ok && mf_matrix_array_bytes(h, name, &bytes) == MF_OK && bytes == count * sizeof(T)) {
        if (bytes && mf_matrix_export(h, name, p, bytes) != MF_OK) ok = false;
    } else {
        ok = false;
    }
    return p;
}

void release_host(Tile_matrix *M)
{
    void *ptrs[] = {M->tile_ptr,      M->tile_columnidx,   M->tile_nnz,     M->Format,        M->blknnz,
                    M->blknnznnz,     M->tilewidth,        M->csr_offset,   M->csrptr_offset, M->Blockcsr_Val,
                    M->Blockcsr_Val_Low, M->Tile_csr_Col,  M->Blockcsr_Ptr, M->csr_compressedIdx};
    for (void *p : ptrs) free(p);
}

}  // namespace

extern "C" {

void Tile_create(Tile_matrix *matrix, int rowA, int colA, int nnzA, int *csrRowPtrA, int *csrColIdxA,
                 double *csrValA, float *csrValA_Low)
{
    (void)nnzA;  // the entries are rowptr[0] .. rowptr[rowA], as in the reference
    if (!matrix) return;
    memset(matrix, 0, sizeof(*matrix));
    mf_matrix h = nullptr;
    if (mf_matrix_create(rowA, colA, csrRowPtrA, csrColIdxA, csrValA, csrValA_Low, 0, nullptr, &h) != MF_OK) {
        fprintf(stderr, "Tile_create: %s\n", mf_last_error());
        return;
    }
    mf_matrix_info inf;
    mf_matrix_get_info(h, &inf);
    const size_t T = (size_t)inf.tilenum, nnz = (size_t)inf.csrsize;
    bool ok = true;
    Tile_matrix &M = *matrix;
    M.tile_ptr = export_array<int>(h, "tile_ptr", (size_t)inf.tilem + 1, ok);
    M.tile_columnidx = export_array<int>(h, "tile_columnidx", T, ok);
    M.tile_nnz = export_array<int>(h, "tile_nnz", T + 1, ok);
    M.blknnz = export_array<int>(h, "blknnz", T + 1, ok);
    M.blknnznnz = export_array<unsigned char>(h, "blknnznnz", T + 1, ok);
    M.csr_offset = export_array<int>(h, "csr_offset", T + 1, ok);
    M.csrptr_offset = export_array<int>(h, "csrptr_offset", T + 1, ok);
    M.Blockcsr_Val = export_array<double>(h, "Blockcsr_Val", nnz, ok);
    M.Blockcsr_Val_Low = export_array<float>(h, "Blockcsr_Val_Low", nnz, ok);
    M.Tile_csr_Col = export_array<unsigned char>(h, "Tile_csr_Col", nnz, ok);
    M.Blockcsr_Ptr = export_array<unsigned char>(h, "Blockcsr_Ptr", (size_t)inf.csrptrlen, ok);
    M.csr_compressedIdx = (unsigned char *)calloc((nnz + 1) / 2 + 1, 1);
    M.Format = (char *)calloc(T + 1, 1);
    M.tilewidth = (char *)calloc(T + 1, 1);
    if (!ok || !M.csr_compressedIdx || !M.Format || !M.tilewidth) {
        fprintf(stderr, "Tile_create: copying the tiles to the host failed: %s\n", mf_last_error());
        release_host(&M);
        mf_matrix_destroy(h);
        memset(matrix, 0, sizeof(*matrix));
        return;
    }
    M.tilem = inf.tilem;
    M.tilen = inf.tilen;
    M.tilenum = inf.tilenum;
    M.csrsize = inf.csrsize;
    M.csrptrlen = inf.csrptrlen;
    M.mf_handle = h;
}

void Tile_destroy(Tile_matrix *matrix)
{
    if (!matrix) return;
    release_host(matrix);
    if (matrix->mf_handle) mf_matrix_destroy((mf_matrix)matrix->mf_handle);
    memset(matrix, 0, sizeof(*matrix));
}

void blockspmv_cpu(Tile_matrix *matrix, int *ptroffset1, int *ptroffset2, int *rowblkblock,
                   unsigned int **blkcoostylerowidx, int **blkcoostylerowidx_colstart,
                   int **blkcoostylerowidx_colstop, int rowA, int colA, int nnzA, int *csrRowPtrA,
                   int *csrColIdxA, double *csrValA, double *x, double *y, double *y_golden)
{
    (void)nnzA;
    (void)y_golden;  // unused by the reference as well
    if (rowblkblock) *rowblkblock = -1;
    if (!matrix || !rowblkblock || !blkcoostylerowidx || !blkcoostylerowidx_colstart || !blkcoostylerowidx_colstop) {
        fprintf(stderr, "blockspmv_cpu: null argument\n");
        return;
    }
    mf_matrix h = (mf_matrix)matrix->mf_handle;
    bool own = false;
    if (!h) {  // a Tile_matrix not made by this Tile_create: build from the CSR
        if (mf_matrix_create(rowA, colA, csrRowPtrA, csrColIdxA, csrValA, nullptr, 0, nullptr, &h) != MF_OK) {
            fprintf(stderr, "blockspmv_cpu: %s\n", mf_last_error());
            return;
        }
        own = true;
    }
    mf_matrix_info inf;
    mf_matrix_get_info(h, &inf);
    const int T = inf.tilenum, R = inf.rowblkblock;
    bool ok = true;
    unsigned int *ri = export_array<unsigned int>(h, "rowblkblock_rowidx", (size_t)R, ok);
    int *cs = export_array<int>(h, "rowblkblock_colstart", (size_t)R, ok);
    int *ce = export_array<int>(h, "rowblkblock_colstop", (size_t)R, ok);
    if (ok && ptroffset1 && T) ok = mf_matrix_export(h, "ptroffset1", ptroffset1, sizeof(int) * T) == MF_OK;
    if (ok && ptroffset2 && T) ok = mf_matrix_export(h, "ptroffset2", ptroffset2, sizeof(int) * T) == MF_OK;
    // y = A x with the columns the struct's csr_compressedIdx holds
    const size_t ny = (size_t)inf.tilem * MF_TILE, nx = (size_t)inf.tilen * MF_TILE;
    const size_t ncidx = ((size_t)inf.csrsize + 1) / 2;
    double *dx = nullptr, *dy = nullptr;
    unsigned char *dc = nullptr;
    if (ok && y && x && matrix->csr_compressedIdx) {
        ok = cudaMalloc(&dx, sizeof(double) * (nx + 1)) == cudaSuccess &&
             cudaMalloc(&dy, sizeof(double) * (ny + 1)) == cudaSuccess &&
             cudaMalloc(&dc, ncidx + 1) == cudaSuccess;
        // x holds tilen*16 readable entries in the reference; the columns
        // past colA meet zeros here
        if (ok) ok = cudaMemset(dx, 0, sizeof(double) * (nx + 1)) == cudaSuccess &&
                     cudaMemset(dy, 0, sizeof(double) * (ny + 1)) == cudaSuccess &&
                     cudaMemcpy(dx, x, sizeof(double) * (size_t)colA, cudaMemcpyHostToDevice) == cudaSuccess &&
                     cudaMemcpy(dc, matrix->csr_compressedIdx, ncidx, cudaMemcpyHostToDevice) == cudaSuccess;
        if (ok) ok = mf::spmv_fp64_cidx(h->v, dc, dx, dy, 0) == MF_OK;
        if (ok) ok = cudaMemcpy(y, dy, sizeof(double) * (size_t)inf.rows, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dc);
    if (own) mf_matrix_destroy(h);
    if (!ok) {
        fprintf(stderr, "blockspmv_cpu: %s\n", mf_last_error());
        free(ri);
        free(cs);
        free(ce);
        return;
    }
    *rowblkblock = R;
    *blkcoostylerowidx = ri;
    *blkcoostylerowidx_colstart = cs;
    *blkcoostylerowidx_colstop = ce;
}

}  // extern "C"
