// main-bicg / main-bicg-mixed: the reference's BiCGSTAB drivers
// (src/main-bicg.cu:1696-1726, src/main-bicg-mixed.cu:2168-2193).  Reads a
// Matrix Market or binary CSR file, x = 0, and calls the BiCGSTAB entry point the
// reference picks by nnz; the entry point sets rhs to the row sums of A.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Mille-feuille-bicg.h"
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
    std::vector<double> x1((size_t)m + 1, 0.0), rhs1((size_t)m + 1, 1.0);
#ifdef MF_CLI_MIXED
    bicgstab(RowPtr, ColIdx, Val, rhs1.data(), x1.data(), nnzR, filename, m);
#else
    if (nnzR < 10000)
        bicgstab_inc(RowPtr, ColIdx, Val, rhs1.data(), x1.data(), nnzR, filename, m);
    else if (nnzR < 100000)
        bicgstab_sync(RowPtr, ColIdx, Val, rhs1.data(), x1.data(), nnzR, filename, m);
    else
        bicgstab(RowPtr, ColIdx, Val, rhs1.data(), x1.data(), nnzR, filename, m);
#endif
    mf_free_host(RowPtr);
    mf_free_host(ColIdx);
    mf_free_host(Val);
    return 0;
}
