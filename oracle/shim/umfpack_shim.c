/* ORACLE TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * CPU implementation behind oracle/shim/umfpack.h.  The reference falls back
 * to UMFPACK's unsymmetric LU when A + delta*I stays indefinite
 * (src/speigs_core.c:975-984) and applies it per Lanczos step (:111-115).
 * Here the "LU" is LAPACK's dense dgetrf/dgetrs on the full matrix as stored
 * (both triangles), which is exact enough for the reference's own indefinite
 * test cases (n = 1,728) and is refused above 20,000 rows.
 */
#include "umfpack.h"

#include <stdlib.h>
#include <string.h>

typedef int blas_int;
#ifndef BLASNAME
#define BLASNAME(x) x##_
#endif
extern void BLASNAME(dgetrf)(blas_int *, blas_int *, double *, blas_int *, blas_int *, blas_int *);
extern void BLASNAME(dgetrs)(const char *, blas_int *, blas_int *, const double *, blas_int *,
                             const blas_int *, double *, blas_int *, blas_int *);

typedef struct { int64_t n; } shim_symbolic;
typedef struct { int64_t n; double *LU; blas_int *ipiv; } shim_numeric;

void umfpack_dl_defaults(double Control[UMFPACK_CONTROL]) {
    for (int i = 0; i < UMFPACK_CONTROL; i++) Control[i] = 0.0;
}

int umfpack_dl_symbolic(int64_t n_row, int64_t n_col, const int64_t *Ap, const int64_t *Ai,
                        const double *Ax, void **Symbolic, const double *Control, double *Info) {
    (void)Ap; (void)Ai; (void)Ax; (void)Control; (void)Info;
    if (n_row != n_col || n_row <= 0 || n_row > 20000) return UMFPACK_ERROR_invalid_matrix;
    shim_symbolic *S = (shim_symbolic *)malloc(sizeof *S);
    if (!S) return UMFPACK_ERROR_out_of_memory;
    S->n = n_row;
    *Symbolic = S;
    return UMFPACK_OK;
}

int umfpack_dl_numeric(const int64_t *Ap, const int64_t *Ai, const double *Ax, void *Symbolic,
                       void **Numeric, const double *Control, double *Info) {
    (void)Control; (void)Info;
    shim_symbolic *S = (shim_symbolic *)Symbolic;
    int64_t n = S->n;
    shim_numeric *N = (shim_numeric *)calloc(1, sizeof *N);
    if (!N) return UMFPACK_ERROR_out_of_memory;
    N->n = n;
    N->LU = (double *)calloc((size_t)(n * n), sizeof(double));
    N->ipiv = (blas_int *)malloc((size_t)n * sizeof(blas_int));
    if (!N->LU || !N->ipiv) { free(N->LU); free(N->ipiv); free(N); return UMFPACK_ERROR_out_of_memory; }
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) N->LU[Ai[q] + c * n] += Ax[q];
    blas_int bn = (blas_int)n, info = 0;
    BLASNAME(dgetrf)(&bn, &bn, N->LU, &bn, N->ipiv, &info);
    *Numeric = N;
    return info > 0 ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

int umfpack_dl_solve(int sys, const int64_t *Ap, const int64_t *Ai, const double *Ax, double *X,
                     const double *B, void *Numeric, const double *Control, double *Info) {
    (void)sys; (void)Ap; (void)Ai; (void)Ax; (void)Control; (void)Info;
    shim_numeric *N = (shim_numeric *)Numeric;
    blas_int bn = (blas_int)N->n, one = 1, info = 0;
    memcpy(X, B, (size_t)N->n * sizeof(double));
    BLASNAME(dgetrs)("N", &bn, &one, N->LU, &bn, N->ipiv, X, &bn, &info);
    return info < 0 ? UMFPACK_ERROR_invalid_matrix : UMFPACK_OK;
}

void umfpack_dl_free_symbolic(void **Symbolic) {
    if (Symbolic && *Symbolic) { free(*Symbolic); *Symbolic = NULL; }
}

void umfpack_dl_free_numeric(void **Numeric) {
    if (!Numeric || !*Numeric) return;
    shim_numeric *N = (shim_numeric *)*Numeric;
    free(N->LU); free(N->ipiv); free(N);
    *Numeric = NULL;
}
