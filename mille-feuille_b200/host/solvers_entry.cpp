// solvers_entry.cpp -- the reference's solve entry points (cg_solve_*,
// bicgstab*) with their signatures and side effects, over libmf.
//
// Compiled twice: MF_SHIM_MIXED=0 gives libmf_solvers.so (the FP64 drivers,
// src/main-cg.cu and src/main-bicg.cu), MF_SHIM_MIXED=1 gives
// libmf_solvers_mixed.so (src/main-cg-mixed.cu, src/main-bicg-mixed.cu).
// The contract of each call is written in Mille-feuille-cg.h and
// Mille-feuille-bicg.h.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Mille-feuille-bicg.h"
#include "Mille-feuille-cg.h"
#include "mf.h"

#ifndef MF_SHIM_MIXED
#define MF_SHIM_MIXED 0
#endif

namespace {

constexpr int TILE = 16;

// Rows [0, n) and columns [0, n) of a CSR matrix, entry order kept.
struct Lead {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    std::vector<float> vl;
};

Lead leading_block(const int *RowPtr, const int *ColIdx, const double *Val, const float *Val_Low, int n)
{
    Lead L;
    L.n = n;
    L.rp.assign((size_t)n + 1, 0);
    for (int i = 0; i < n; i++) {
        for (int j = RowPtr[i]; j < RowPtr[i + 1]; j++) {
            if (ColIdx[j] < 0 || ColIdx[j] >= n) continue;
            L.ci.push_back(ColIdx[j]);
            L.v.push_back(Val[j]);
            if (Val_Low) L.vl.push_back(Val_Low[j]);
        }
        L.rp[(size_t)i + 1] = (int)L.ci.size();
    }
    return L;
}

bool env_double(const char *name, double *out)
{
    const char *s = getenv(name);
    if (!s || !*s) return false;
    char *end = nullptr;
    const double v = strtod(s, &end);
    if (end == s) return false;
    *out = v;
    return true;
}

// Iteration count / tolerance / policy of one call.
void configure(mf_solve_opts &o, int fixed_iters, bool bicg)
{
    mf_solve_opts_default(&o);
    double t = 0, k = 0;
    const bool have_tol = env_double("MF_SHIM_TOL", &t) && t > 0;
    const bool have_k = env_double("MF_SHIM_MAXITER", &k) && k >= 0;
    o.tol = have_tol ? t : -1.0;
    o.maxiter = have_k ? (int)k : (have_tol ? 20000 : fixed_iters);
    o.policy = MF_POLICY_FP64;
    if (MF_SHIM_MIXED) {
        o.policy = bicg ? MF_POLICY_STATIC : MF_POLICY_RULE;
        const char *p = getenv("MF_SHIM_POLICY");
        if (p && !strcmp(p, "static")) o.policy = MF_POLICY_STATIC;
        if (p && !strcmp(p, "rule")) o.policy = MF_POLICY_RULE;
        if (p && !strcmp(p, "rule_scaled")) o.policy = MF_POLICY_RULE_SCALED;
        if (p && !strcmp(p, "static_fp16")) o.policy = MF_POLICY_STATIC_FP16;
        if (p && !strcmp(p, "learned")) o.policy = MF_POLICY_LEARNED;
    }
}

double norm2(const double *v, int n)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += v[i] * v[i];
    return std::sqrt(s);
}

void append_csv(const char *path, const char *filename, int count, double ms, int nnzR, double l2, double last)
{
    FILE *f = fopen(path, "a");
    if (!f) {
        printf("open error!\n");
        return;
    }
    fprintf(f, "%s,%d,%.3f,%d,%e,%e\n", filename ? filename : "", count, ms, nnzR, l2, last);
    fclose(f);
}

// Builds the matrix, attaches a learned policy when one is asked for, solves.
mf_status solve(bool bicg, const Lead &L, const double *b, double *x, const mf_solve_opts &o, mf_solve_report &rep)
{
    memset(&rep, 0, sizeof(rep));
    mf_matrix m = nullptr;
    mf_status st = mf_matrix_create(L.n, L.n, L.rp.data(), L.ci.empty() ? nullptr : L.ci.data(),
                                    L.v.empty() ? nullptr : L.v.data(), L.vl.empty() ? nullptr : L.vl.data(), 0,
                                    nullptr, &m);
    if (st != MF_OK) return st;
    mf_learned pol = nullptr;
    if (o.policy == MF_POLICY_LEARNED) {
        const char *pf = getenv("MF_POLICY_FILE");
        st = pf ? mf_policy_load(pf, &pol) : MF_ERR_INVALID_ARG;
        if (st == MF_OK) st = mf_matrix_attach_policy(m, pol);
        if (st != MF_OK && !pf) fprintf(stderr, "MF_SHIM_POLICY=learned needs MF_POLICY_FILE\n");
    }
    if (st == MF_OK) st = bicg ? mf_bicgstab_solve_host(m, b, x, &o, &rep) : mf_cg_solve_host(m, b, x, &o, &rep);
    mf_matrix_destroy(m);
    if (pol) mf_policy_destroy(pol);
    return st;
}

void cg_entry(int fixed_iters, int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n,
              int *iter, char *filename, int nnzR)
{
    if (n <= 0 || !RowPtr || !x || !b) {
        fprintf(stderr, "cg_solve: invalid arguments\n");
        return;
    }
    memset(x, 0, sizeof(double) * (size_t)n);
    const int rowA = n / TILE * TILE;
    const Lead L = leading_block(RowPtr, ColIdx, Val, Val_Low, rowA);
    mf_solve_opts o;
    configure(o, fixed_iters, false);
    mf_solve_report rep;
    const mf_status st = rowA ? solve(false, L, b, x, o, rep) : MF_OK;
    if (st != MF_OK && st != MF_ERR_NOT_CONVERGED) fprintf(stderr, "cg_solve: %s\n", mf_last_error());
    if (iter) *iter = rep.iterations;
    const double ms100 = rep.iterations ? rep.kernel_ms * 100.0 / rep.iterations : 0.0;
    printf("time_cg=%lf ms\n", ms100);
    const double nb = norm2(b, rowA);
    append_csv("data/cg_performance.csv", filename, 100, ms100, nnzR, rep.relres_true, rep.relres * nb);
}

int bicg_entry(int fixed_iters, int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
               char *filename, int n)
{
    if (n <= 0 || !RowPtr || !rhs || !x) {
        fprintf(stderr, "bicgstab: invalid arguments\n");
        return 1;
    }
    const int rowA = n / TILE * TILE;
    for (int i = 0; i < rowA; i++) {
        double s = 0;
        for (int j = RowPtr[i]; j < RowPtr[i + 1]; j++) s += Val[j];
        rhs[i] = s;
    }
    const Lead L = leading_block(RowPtr, ColIdx, Val, nullptr, rowA);
    // initial guess x0: solve A e = rhs - A x0, then x = x0 + e
    std::vector<double> x0(x, x + rowA), r0(rhs, rhs + rowA), e((size_t)rowA, 0.0);
    bool nonzero_x0 = false;
    for (int i = 0; i < rowA; i++) nonzero_x0 |= (x0[i] != 0.0);
    if (nonzero_x0)
        for (int i = 0; i < rowA; i++)
            for (int j = L.rp[i]; j < L.rp[i + 1]; j++) r0[i] -= L.v[j] * x0[L.ci[j]];
    mf_solve_opts o;
    configure(o, fixed_iters, true);
    mf_solve_report rep;
    const mf_status st = rowA ? solve(true, L, r0.data(), e.data(), o, rep) : MF_OK;
    if (st != MF_OK && st != MF_ERR_NOT_CONVERGED) fprintf(stderr, "bicgstab: %s\n", mf_last_error());
    for (int i = 0; i < rowA; i++) x[i] = x0[i] + e[i];
    double l2 = rep.relres_true;
    if (nonzero_x0) {  // relative to rhs, not to the correction's right-hand side
        double rr = 0;
        for (int i = 0; i < rowA; i++) {
            double ax = 0;
            for (int j = L.rp[i]; j < L.rp[i + 1]; j++) ax += L.v[j] * x[L.ci[j]];
            rr += (rhs[i] - ax) * (rhs[i] - ax);
        }
        const double nb = norm2(rhs, rowA);
        l2 = nb > 0 ? std::sqrt(rr) / nb : std::sqrt(rr);
    }
    const double ms50 = rep.iterations ? rep.kernel_ms * 50.0 / rep.iterations : 0.0;
    printf("time_bicg=%lf ms\n", ms50);
    append_csv("data/bicg_performance.csv", filename, 50, ms50, nnzR, l2, rep.relres);
    return (st != MF_OK && st != MF_ERR_NOT_CONVERGED) || rep.iterations >= o.maxiter ? 1 : 0;
}

}  // namespace

extern "C" {

void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                  int maxiter, double threshold, char *filename, int nnzR, int ori)
{
    (void)maxiter, (void)threshold, (void)ori;
    cg_entry(100, RowPtr, ColIdx, Val, Val_Low, x, b, n, iter, filename, nnzR);
}

void cg_solve_sync(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                   int maxiter, double threshold, char *filename, int nnzR, int ori)
{
    (void)maxiter, (void)threshold, (void)ori;
    cg_entry(100, RowPtr, ColIdx, Val, Val_Low, x, b, n, iter, filename, nnzR);
}

void cg_solve_reduce(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                     int maxiter, double threshold, char *filename, int nnzR, int ori)
{
    (void)maxiter, (void)threshold, (void)ori;
    cg_entry(10000, RowPtr, ColIdx, Val, Val_Low, x, b, n, iter, filename, nnzR);
}

int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n)
{
    return bicg_entry(10000, RowPtr, ColIdx, Val, rhs, x, nnzR, filename, n);
}

int bicgstab_sync(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n)
{
    return bicg_entry(50, RowPtr, ColIdx, Val, rhs, x, nnzR, filename, n);
}

int bicgstab_inc(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n)
{
    return bicg_entry(50, RowPtr, ColIdx, Val, rhs, x, nnzR, filename, n);
}

}  // extern "C"
