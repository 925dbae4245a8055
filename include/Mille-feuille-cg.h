/*
 * Mille-feuille-cg.h -- the reference's CG solve entry points, same names
 * and signatures, served by libmf_solvers.so (FP64) and
 * libmf_solvers_mixed.so (tile mixed precision with the partial-convergence
 * rule, FP64 refinement).
 *
 *   cg_solve_reduce  src/main-cg.cu:6       multi-kernel CG, 10000 iterations
 *   cg_solve_sync    src/main-cg.cu:379     persistent CG, 100 iterations
 *   cg_solve_inc     src/main-cg.cu:1071    persistent CG, 100 iterations
 *                    src/main-cg-mixed.cu:2238 (mixed precision)
 *
 * Behaviour kept from the reference:
 *   - rows are truncated to n / 16 * 16; x (n entries, host) is zeroed on
 *     entry and receives the solution; b (host) is read, never written;
 *   - iter, maxiter and threshold are ignored; the iteration count is fixed
 *     (100, or 10000 for cg_solve_reduce);
 *   - "time_cg=<ms> ms" is printed and one line
 *     "<filename>,100,<ms per 100 iterations>,<nnzR>,<l2_norm>,<sqrt(snew)>"
 *     is appended to data/cg_performance.csv (relative to the working
 *     directory; "open error!" is printed when it cannot be opened).
 * Defined here where the reference is undefined or silent:
 *   - the system solved is the leading (n/16*16)^2 block: entries in columns
 *     at or past the truncated row count meet the zero padding of the
 *     direction vector in the reference, and are dropped here;
 *   - l2_norm is the FP64 true relative residual ||b - A x|| / ||b||,
 *     sqrt(snew) the recurrence residual norm ||r||;
 *   - *iter (when not NULL) receives the iterations run;
 *   - failures print "cg_solve: <message>" to stderr and leave x at the
 *     last iterate (zeros when nothing ran).
 * Environment overrides (both optional): MF_SHIM_TOL=<t> stops at relative
 * residual t instead of the fixed count, MF_SHIM_MAXITER=<k> sets the
 * iteration count (or the cap under MF_SHIM_TOL).  In the mixed library
 * MF_SHIM_POLICY=static|rule|learned picks the precision policy (rule by
 * default; learned needs MF_POLICY_FILE=<file written by mf_policy_save>).
 */
#ifndef MILLE_FEUILLE_CG_H
#define MILLE_FEUILLE_CG_H

#ifdef __cplusplus
extern "C" {
#endif

void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                  int maxiter, double threshold, char *filename, int nnzR, int ori);
void cg_solve_sync(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                   int maxiter, double threshold, char *filename, int nnzR, int ori);
void cg_solve_reduce(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                     int maxiter, double threshold, char *filename, int nnzR, int ori);

#ifdef __cplusplus
}
#endif
#endif
