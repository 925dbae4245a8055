// main-cg / main-cg-mixed: the reference's CG drivers (src/main-cg.cu:1630-1673,
// src/main-cg-mixed.cu:3006-3042).  Reads a Matrix Market or binary CSR file, truncates the
// rows to a multiple of 16, sets b = A * ones and calls the CG entry point
// the reference picks by nnz (main-cg) or cg_solve_inc (main-cg-mixed).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Mille-feuille-cg.h"
#include "mf.h"

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s matrix.mtx|matrix.cbd\n", argv[0]);
        return 1;
    }
    char *filename = argv[1];
    int m = 0, n = 0, nnzR = 0, sym = 0;
    int *RowPtr = nullptr, *ColIdx = nullptr;
    double *Val = nullptr;
    // .mtx or .cbd by extension, as the reference's read_Dmatrix_32, which
    // announces a binary file on stdout
    const size_t flen = strlen(filename);
    if (flen >= 3 && !strcmp(filename + flen - 3, "cbd")) printf("read binary file %s\n", filename);
    if (mf_read_matrix(filename, &m, &n, &nnzR, &RowPtr, &ColIdx, &Val, &sym) != MF_OK) {
        fprintf(stderr, "%s\n", mf_last_error());
        return 1;
    }
    if (m != n) {
#ifndef MF_CLI_MIXED
        printf("unequal\n");
#endif
        return 0;
    }
    std::vector<float> Val_Low((size_t)nnzR + 1);
    for (int i = 0; i < nnzR; i++) Val_Low[i] = (float)Val[i];
    const int ori = n;
    n = n / 16 * 16;
    // b = A * ones over the truncated rows (every column of those rows)
    std::vector<double> X((size_t)n + 1, 1.0), Y((size_t)n + 1, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = RowPtr[i]; j < RowPtr[i + 1]; j++) Y[i] += Val[j] * 1.0;
    int iter = 0;
#ifdef MF_CLI_MIXED
    cg_solve_inc(RowPtr, ColIdx, Val, Val_Low.data(), X.data(), Y.data(), n, &iter, 10, 1e-5, filename, nnzR, ori);
#else
    if (nnzR < 10000)
        cg_solve_inc(RowPtr, ColIdx, Val, Val_Low.data(), X.data(), Y.data(), n, &iter, 10, 1e-5, filename, nnzR, ori);
    else if (nnzR < 100000)
        cg_solve_sync(RowPtr, ColIdx, Val, Val_Low.data(), X.data(), Y.data(), n, &iter, 10, 1e-5, filename, nnzR, ori);
    else
        cg_solve_reduce(RowPtr, ColIdx, Val, Val_Low.data(), X.data(), Y.data(), n, &iter, 10, 1e-5, filename, nnzR,
                        ori);
#endif
    mf_free_host(RowPtr);
    mf_free_host(ColIdx);
    mf_free_host(Val);
    return 0;
}
