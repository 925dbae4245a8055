/*
 * Mille-feuille-bicg.h -- the reference's BiCGSTAB entry points, same names
 * and signatures, served by libmf_solvers.so (FP64) and
 * libmf_solvers_mixed.so (tile mixed precision, FP64 refinement).
 *
 *   bicgstab_sync  src/main-bicg.cu:13      persistent BiCGSTAB, 50 iterations
 *   bicgstab_inc   src/main-bicg.cu:711     persistent BiCGSTAB, 50 iterations
 *   bicgstab       src/main-bicg.cu:1336    multi-kernel BiCGSTAB, 10000 iterations
 *                  src/main-bicg-mixed.cu:1355 (mixed precision)
 *
 * Behaviour kept from the reference:
 *   - n is the row count; rows are truncated to n / 16 * 16;
 *   - rhs (host) is overwritten with the row sums of A (A times ones, over
 *     all columns), which is the right-hand side solved for;
 *   - x (host) is the initial guess;
 *   - the iteration count is fixed (50, or 10000 for bicgstab);
 *   - "time_bicg=<ms> ms" is printed and one line
 *     "<filename>,50,<ms per 50 iterations>,<nnzR>,<l2_norm>,<relres>"
 *     is appended to data/bicg_performance.csv;
 *   - the return value is 1 when the iteration limit was reached, else 0.
 * Defined here where the reference is undefined or silent:
 *   - the leading (n/16*16)^2 block is solved (as for CG);
 *   - x receives the solution (the reference leaves it unchanged);
 *   - l2_norm is the FP64 true relative residual, relres the recurrence's;
 *   - failures print "bicgstab: <message>" to stderr and return 1.
 * Environment overrides as for the CG entry points (MF_SHIM_TOL,
 * MF_SHIM_MAXITER; MF_SHIM_POLICY=static in the mixed library).
 */
#ifndef MILLE_FEUILLE_BICG_H
#define MILLE_FEUILLE_BICG_H

#ifdef __cplusplus
extern "C" {
#endif

int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n);
int bicgstab_sync(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n);
int bicgstab_inc(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n);

#ifdef __cplusplus
}
#endif
#endif
