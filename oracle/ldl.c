/*
 * oracle/ldl.c -- TEST INFRASTRUCTURE, not the product.
 *
 * Sparse LDL^T with the QDLDL calling convention (QDLDL_etree, QDLDL_factor,
 * QDLDL_solve), FP32 values and int32 indices, as the reference builds qdldl
 * (README.md:14-19: QDLDL_FLOAT=true, QDLDL_LONG=false) and calls it
 * (toplevel.cuh:207, qdldl_helper.cuh:125,136).  The qdldl submodule
 * (osqp/qdldl, unpinned, .gitmodules:7-9) is absent from the reference tree;
 * this is written from the published up-looking elimination-tree algorithm
 * (T. A. Davis, "Algorithm 849: A concise sparse Cholesky factorization
 * package", ACM TOMS 31(4), 2005), without pivoting or permutation, like the
 * reference's call.  The input is the upper triangle in CSC form.  An LDL^T
 * without permutation of a definite matrix is unique, so any correct
 * implementation agrees with qdldl up to rounding.
 */
#include <stdint.h>
#include <stdlib.h>

typedef int32_t QDLDL_int;
typedef float QDLDL_float;
typedef unsigned char QDLDL_bool;

/* elimination tree and column counts; returns sum of Lnz or -1 */
QDLDL_int QDLDL_etree(const QDLDL_int n, const QDLDL_int *Ap, const QDLDL_int *Ai, QDLDL_int *work,
                      QDLDL_int *Lnz, QDLDL_int *etree)
{
    for (QDLDL_int i = 0; i < n; ++i) { work[i] = 0; Lnz[i] = 0; etree[i] = -1; }
    for (QDLDL_int j = 0; j < n; ++j) {
        work[j] = j;
        for (QDLDL_int p = Ap[j]; p < Ap[j + 1]; ++p) {
            QDLDL_int i = Ai[p];
            if (i > j) return -1; /* not upper triangular */
            while (work[i] != j) {
                if (etree[i] == -1) etree[i] = j;
                Lnz[i]++;
                work[i] = j;
                i = etree[i];
            }
        }
    }
    QDLDL_int sum = 0;
    for (QDLDL_int i = 0; i < n; ++i) sum += Lnz[i];
    return sum;
}

/* numeric factorisation (up-looking, one row of L per step); returns the
 * number of positive entries of D, or -1 on a zero pivot */
QDLDL_int QDLDL_factor(const QDLDL_int n, const QDLDL_int *Ap, const QDLDL_int *Ai, const QDLDL_float *Ax,
                       QDLDL_int *Lp, QDLDL_int *Li, QDLDL_float *Lx, QDLDL_float *D, QDLDL_float *Dinv,
                       const QDLDL_int *Lnz, const QDLDL_int *etree, QDLDL_bool *bwork, QDLDL_int *iwork,
                       QDLDL_float *fwork)
{
    QDLDL_int *flag = iwork, *pattern = iwork + n, *cnt = iwork + 2 * n;
    QDLDL_float *y = fwork;
    (void)bwork;
    Lp[0] = 0;
    for (QDLDL_int i = 0; i < n; ++i) Lp[i + 1] = Lp[i] + Lnz[i];
    QDLDL_int npos = 0;
    for (QDLDL_int k = 0; k < n; ++k) {
        y[k] = 0;
        QDLDL_int top = n;
        flag[k] = k;
        cnt[k] = 0;
        for (QDLDL_int p = Ap[k]; p < Ap[k + 1]; ++p) {
            QDLDL_int i = Ai[p];
            y[i] += Ax[p];
            QDLDL_int len = 0;
            for (; flag[i] != k; i = etree[i]) { pattern[len++] = i; flag[i] = k; }
            while (len > 0) pattern[--top] = pattern[--len];
        }
        D[k] = y[k];
        y[k] = 0;
        for (; top < n; ++top) {
            QDLDL_int i = pattern[top];
            QDLDL_float yi = y[i];
            y[i] = 0;
            QDLDL_int p2 = Lp[i] + cnt[i];
            for (QDLDL_int p = Lp[i]; p < p2; ++p) y[Li[p]] -= Lx[p] * yi;
            QDLDL_float lki = yi / D[i];
            D[k] -= lki * yi;
            Li[p2] = k;
            Lx[p2] = lki;
            cnt[i]++;
        }
        if (D[k] == 0) return -1;
        if (D[k] > 0) npos++;
        Dinv[k] = 1 / D[k];
    }
    return npos;
}

/* solve L D L^T x = b in place (x holds b on entry) */
void QDLDL_solve(const QDLDL_int n, const QDLDL_int *Lp, const QDLDL_int *Li, const QDLDL_float *Lx,
                 const QDLDL_float *Dinv, QDLDL_float *x)
{
    for (QDLDL_int j = 0; j < n; ++j)
        for (QDLDL_int p = Lp[j]; p < Lp[j + 1]; ++p) x[Li[p]] -= Lx[p] * x[j];
    for (QDLDL_int j = 0; j < n; ++j) x[j] *= Dinv[j];
    for (QDLDL_int j = n - 1; j >= 0; --j)
        for (QDLDL_int p = Lp[j]; p < Lp[j + 1]; ++p) x[j] -= Lx[p] * x[Li[p]];
}

/* qdldl_solve_schur (qdldl_helper.cuh:62-180) with its allocations
 * (toplevel.cuh:183-212) folded in: etree, factor, solve. */
int orc_ldl_solve(int n, const int32_t *Ap, const int32_t *Ai, const float *Ax, const float *b, float *x)
{
    QDLDL_int *iwork = malloc(sizeof(QDLDL_int) * 3 * n), *Lnz = malloc(sizeof(QDLDL_int) * n),
              *etree = malloc(sizeof(QDLDL_int) * n), *Lp = malloc(sizeof(QDLDL_int) * (n + 1));
    QDLDL_float *D = malloc(sizeof(QDLDL_float) * n), *Dinv = malloc(sizeof(QDLDL_float) * n),
                *fwork = malloc(sizeof(QDLDL_float) * n);
    QDLDL_bool *bwork = malloc(n);
    int rc = 0;
    QDLDL_int sum = QDLDL_etree(n, Ap, Ai, iwork, Lnz, etree);
    if (sum < 0) { rc = -1; goto out; }
    {
        QDLDL_int *Li = malloc(sizeof(QDLDL_int) * (sum > 0 ? sum : 1));
        QDLDL_float *Lx = malloc(sizeof(QDLDL_float) * (sum > 0 ? sum : 1));
        if (QDLDL_factor(n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, Lnz, etree, bwork, iwork, fwork) < 0) rc = -1;
        else {
            for (int i = 0; i < n; ++i) x[i] = b[i];
            QDLDL_solve(n, Lp, Li, Lx, Dinv, x);
        }
        free(Li); free(Lx);
    }
out:
    free(iwork); free(Lnz); free(etree); free(Lp); free(D); free(Dinv); free(fwork); free(bwork);
    return rc;
}
