/* ORACLE TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * CPU implementation behind oracle/shim/cholmod.h: the subset of CHOLMOD the
 * reference's src/speigs_core.c calls, so that file can be compiled verbatim
 * and serve as the CPU oracle and the timed CPU baseline.
 *
 *   cholmod_l_norm_sparse  (speigs_core.c:840)  1-norm of the symmetric matrix
 *                                               whose upper triangle is stored
 *   cholmod_l_sdmult       (:82)                y = A x, upper triangle read
 *   cholmod_l_analyze      (:934)               ordering + symbolic analysis
 *   cholmod_l_factorize_p  (:940, :966)         numeric LL^T of A + beta*I,
 *                                               status NOT_POSDEF on failure
 *   cholmod_l_solve2       (:96)                x = A^{-1} b, X/Y/E reused
 *
 * The numeric factorization is a multifrontal supernodal LL^T on the CPU:
 * every front is assembled from A and the children's update matrices and
 * factored with LAPACK/BLAS-3 (dpotrf, dtrsm, dsyrk), which is how CHOLMOD's
 * supernodal module spends its time too.  The ordering and symbolic analysis
 * come from the host analysis that the GPU library uses
 * (sparse-eigs-mex_b200/csrc/host/symbolic.cpp); the ordering only changes
 * rounding, never the eigenpairs, so both sides use the same one.
 */
#include "cholmod.h"
#include "../../sparse-eigs-mex_b200/csrc/host/symbolic.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef int blas_int;
#ifndef BLASNAME
#define BLASNAME(x) x##_
#endif
extern void BLASNAME(dpotrf)(const char *, blas_int *, double *, blas_int *, blas_int *);
extern void BLASNAME(dtrsm)(const char *, const char *, const char *, const char *, blas_int *,
                            blas_int *, const double *, const double *, blas_int *, double *,
                            blas_int *);
extern void BLASNAME(dsyrk)(const char *, const char *, blas_int *, blas_int *, const double *,
                            const double *, blas_int *, const double *, double *, blas_int *);
extern void BLASNAME(dtrsv)(const char *, const char *, const char *, blas_int *, const double *,
                            blas_int *, double *, blas_int *);
extern void BLASNAME(dgemv)(const char *, blas_int *, blas_int *, const double *, const double *,
                            blas_int *, const double *, blas_int *, const double *, double *,
                            blas_int *);

struct cholmod_factor {
    int64_t      n;
    spx_symbolic S;
    int64_t     *rp;     /* full symmetric CSR built from the upper triangle */
    int32_t     *ci;
    double      *cx;
    int64_t     *lxptr;  /* compact r x c panels */
    double      *Lx;
    int          is_factored;
};

int cholmod_l_start(cholmod_common *cc) {
    memset(cc, 0, sizeof *cc);
    cc->supernodal = CHOLMOD_AUTO;
    cc->nmethods = 0;
    cc->postorder = 1;
    cc->status = CHOLMOD_OK;
    return 1;
}

int cholmod_l_finish(cholmod_common *cc) { (void)cc; return 1; }

/* ||A||_1 of the symmetric matrix represented by the upper triangle
 * (stype = 1, as the reference passes at speigs_core.c:836). */
double cholmod_l_norm_sparse(cholmod_sparse *A, int norm, cholmod_common *cc) {
    (void)norm; (void)cc;
    const int64_t *Ap = (const int64_t *)A->p, *Ai = (const int64_t *)A->i;
    const double *Ax = (const double *)A->x;
    int64_t n = (int64_t)A->ncol;
    double *s = (double *)calloc((size_t)n, sizeof(double));
    if (!s) return -1.0;
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t r = Ai[q];
            if (r > c) continue;
            double a = fabs(Ax[q]);
            s[c] += a;
            if (r != c) s[r] += a;
        }
    double m = 0.0;
    for (int64_t c = 0; c < n; c++) if (s[c] > m) m = s[c];
    free(s);
    return m;
}

/* Y = alpha*A*X + beta*Y for the symmetric A of the upper triangle. */
int cholmod_l_sdmult(cholmod_sparse *A, int transpose, double alpha[2], double beta[2],
                     cholmod_dense *X, cholmod_dense *Y, cholmod_common *cc) {
    (void)transpose; (void)cc;
    const int64_t *Ap = (const int64_t *)A->p, *Ai = (const int64_t *)A->i;
    const double *Ax = (const double *)A->x;
    int64_t n = (int64_t)A->ncol;
    const double *x = (const double *)X->x;
    double *y = (double *)Y->x;
    for (int64_t i = 0; i < n; i++) y[i] = (beta[0] == 0.0) ? 0.0 : beta[0] * y[i];
    /* column sweep: the column's own entry and the strictly-upper entries are
     * scattered with x[c]; the transposed contributions to y[c] are gathered
     * into one accumulator and added once per column */
    for (int64_t c = 0; c < n; c++) {
        const double xc = alpha[0] * x[c];
        double yc = 0.0;
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t r = Ai[q];
            if (r > c) continue;
            y[r] += Ax[q] * xc;
            if (r != c) yc += Ax[q] * x[r];
        }
        y[c] += alpha[0] * yc;
    }
    return 1;
}

/* full symmetric CSR (int32 columns) from the upper triangle of a CSC */
static int build_full(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                      int64_t **rp_o, int32_t **ci_o, double **cx_o) {
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!cnt) return 0;
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t r = Ai[q];
            if (r > c) continue;
            cnt[r + 1]++;
            if (r != c) cnt[c + 1]++;
        }
    for (int64_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    int64_t nnz = cnt[n];
    int32_t *ci = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
    double *cx = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
    int64_t *fill = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    if (!ci || !cx || !fill) { free(cnt); free(ci); free(cx); free(fill); return 0; }
    memcpy(fill, cnt, (size_t)n * sizeof(int64_t));
    /* columns visited in increasing order => each row's columns come out sorted */
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t r = Ai[q];
            if (r > c) continue;
            int64_t d = fill[r]++;
            ci[d] = (int32_t)c; cx[d] = Ax[q];
        }
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t r = Ai[q];
            if (r >= c) continue;
            int64_t d = fill[c]++;
            ci[d] = (int32_t)r; cx[d] = Ax[q];
        }
    /* rows now hold lower-part columns after upper-part ones; sort each row */
    for (int64_t i = 0; i < n; i++) {
        for (int64_t a = cnt[i] + 1; a < cnt[i + 1]; a++) {
            int32_t kc = ci[a]; double kx = cx[a]; int64_t b = a - 1;
            while (b >= cnt[i] && ci[b] > kc) { ci[b + 1] = ci[b]; cx[b + 1] = cx[b]; b--; }
            ci[b + 1] = kc; cx[b + 1] = kx;
        }
    }
    free(fill);
    *rp_o = cnt; *ci_o = ci; *cx_o = cx;
    return 1;
}

cholmod_factor *cholmod_l_analyze(cholmod_sparse *A, cholmod_common *cc) {
    int64_t n = (int64_t)A->ncol;
    if (n <= 0 || n > 0x7fffffffLL) { cc->status = -4; return NULL; }
    cholmod_factor *L = (cholmod_factor *)calloc(1, sizeof *L);
    if (!L) { cc->status = -2; return NULL; }
    L->n = n;
    if (!build_full(n, (const int64_t *)A->p, (const int64_t *)A->i, (const double *)A->x,
                    &L->rp, &L->ci, &L->cx)) { free(L); cc->status = -2; return NULL; }
    int ord = (cc->nmethods > 0 && cc->method[0].ordering == CHOLMOD_AMD) ? SPX_ORDER_MINDEG
                                                                         : SPX_ORDER_ND;
    if (spx_analyze((int32_t)n, L->rp, L->ci, ord, &L->S) != 0) {
        free(L->rp); free(L->ci); free(L->cx); free(L); cc->status = -2; return NULL;
    }
    const spx_symbolic *S = &L->S;
    L->lxptr = (int64_t *)malloc((size_t)(S->nsuper + 1) * sizeof(int64_t));
    if (!L->lxptr) { cholmod_l_free_factor(&L, cc); cc->status = -2; return NULL; }
    L->lxptr[0] = 0;
    for (int32_t s = 0; s < S->nsuper; s++) {
        int64_t r = S->rowptr[s + 1] - S->rowptr[s], c = S->sfirst[s + 1] - S->sfirst[s];
        L->lxptr[s + 1] = L->lxptr[s] + r * c;
    }
    cc->status = CHOLMOD_OK;
    return L;
}

/* Multifrontal numeric factorization of A + beta[0]*I. */
int cholmod_l_factorize_p(cholmod_sparse *A, double beta[2], int64_t *fset, size_t fsize,
                          cholmod_factor *L, cholmod_common *cc) {
    (void)A; (void)fset; (void)fsize;
    const spx_symbolic *S = &L->S;
    const int32_t ns = S->nsuper;
    free(L->Lx);
    L->Lx = (double *)malloc((size_t)(L->lxptr[ns] ? L->lxptr[ns] : 1) * sizeof(double));
    double **front = (double **)calloc((size_t)ns, sizeof(double *));
    int32_t *pos = (int32_t *)malloc((size_t)L->n * sizeof(int32_t));
    if (!L->Lx || !front || !pos) { free(front); free(pos); cc->status = -2; return 0; }
    L->is_factored = 0;
    int status = CHOLMOD_OK;
    const double shift = beta ? beta[0] : 0.0;
    for (int32_t s = 0; s < ns && status == CHOLMOD_OK; s++) {
        const int64_t r = S->rowptr[s + 1] - S->rowptr[s];
        const int32_t f = S->sfirst[s], c = S->sfirst[s + 1] - f;
        const int32_t *rows = S->rows + S->rowptr[s];
        double *F = (double *)calloc((size_t)(r * r), sizeof(double));
        if (!F) { status = -2; break; }
        front[s] = F;
        for (int64_t t = 0; t < r; t++) pos[rows[t]] = (int32_t)t;
        for (int32_t jj = 0; jj < c; jj++) {
            int32_t j = f + jj, o = S->perm[j];
            for (int64_t q = L->rp[o]; q < L->rp[o + 1]; q++) {
                int32_t i = S->iperm[L->ci[q]];
                if (i < j) continue;
                F[pos[i] + (int64_t)jj * r] += L->cx[q];
            }
            F[jj + (int64_t)jj * r] += shift;
        }
        for (int32_t q = S->child_ptr[s]; q < S->child_ptr[s + 1]; q++) {
            int32_t ch = S->child_list[q];
            int64_t rc = S->rowptr[ch + 1] - S->rowptr[ch];
            int32_t cc0 = S->sfirst[ch + 1] - S->sfirst[ch];
            const int32_t *rm = S->relmap + S->rowptr[ch];
            double *C = front[ch];
            for (int64_t b = cc0; b < rc; b++) {
                int64_t pb = rm[b];
                for (int64_t a = b; a < rc; a++)
                    F[rm[a] + pb * r] += C[a + b * rc];
            }
            free(C);
            front[ch] = NULL;
        }
        blas_int bc = c, br = (blas_int)r, bm = (blas_int)(r - c), info = 0;
        BLASNAME(dpotrf)("L", &bc, F, &br, &info);
        if (info != 0) { status = CHOLMOD_NOT_POSDEF; break; }
        if (bm > 0) {
            const double one = 1.0, mone = -1.0;
            BLASNAME(dtrsm)("R", "L", "T", "N", &bm, &bc, &one, F, &br, F + c, &br);
            BLASNAME(dsyrk)("L", "N", &bm, &bc, &mone, F + c, &br, &one,
                            F + c + (int64_t)c * r, &br);
        }
        /* keep the r x c panel compactly */
        double *P = L->Lx + L->lxptr[s];
        for (int32_t jj = 0; jj < c; jj++)
            memcpy(P + (int64_t)jj * r, F + (int64_t)jj * r, (size_t)r * sizeof(double));
        if (S->sparent[s] < 0) { free(F); front[s] = NULL; }
    }
    for (int32_t s = 0; s < ns; s++) free(front[s]);
    free(front);
    free(pos);
    if (status == -2) { cc->status = -2; return 0; }
    cc->status = status;
    L->is_factored = (status == CHOLMOD_OK);
    return 1;
}

int cholmod_l_solve2(int sys, cholmod_factor *L, cholmod_dense *B, cholmod_sparse *Bset,
                     cholmod_dense **X_Handle, cholmod_sparse **Xset_Handle,
                     cholmod_dense **Y_Handle, cholmod_dense **E_Handle, cholmod_common *cc) {
    (void)sys; (void)Bset; (void)Xset_Handle;
    if (!L || !L->is_factored) { cc->status = -4; return 0; }
    const spx_symbolic *S = &L->S;
    const int64_t n = L->n;
    if (!*X_Handle) {
        cholmod_dense *X = (cholmod_dense *)calloc(1, sizeof *X);
        if (!X) { cc->status = -2; return 0; }
        X->nrow = X->d = X->nzmax = (size_t)n; X->ncol = 1;
        X->xtype = CHOLMOD_REAL; X->dtype = CHOLMOD_DOUBLE;
        X->x = malloc((size_t)n * sizeof(double));
        if (!X->x) { free(X); cc->status = -2; return 0; }
        *X_Handle = X;
    }
    if (!*Y_Handle) {   /* workspace: permuted vector + one front-length buffer */
        cholmod_dense *Y = (cholmod_dense *)calloc(1, sizeof *Y);
        if (!Y) { cc->status = -2; return 0; }
        Y->nrow = Y->d = Y->nzmax = (size_t)(n + S->max_rows); Y->ncol = 1;
        Y->xtype = CHOLMOD_REAL; Y->dtype = CHOLMOD_DOUBLE;
        Y->x = malloc((size_t)(n + S->max_rows) * sizeof(double));
        if (!Y->x) { free(Y); cc->status = -2; return 0; }
        *Y_Handle = Y;
    }
    (void)E_Handle;
    double *y = (double *)(*Y_Handle)->x, *tmp = y + n;
    const double *b = (const double *)B->x;
    double *x = (double *)(*X_Handle)->x;
    for (int64_t i = 0; i < n; i++) y[i] = b[S->perm[i]];
    const double one = 1.0, zero = 0.0;
    blas_int inc = 1;
    for (int32_t s = 0; s < S->nsuper; s++) {           /* forward: L y = P b */
        const int64_t r = S->rowptr[s + 1] - S->rowptr[s];
        const int32_t f = S->sfirst[s], c = S->sfirst[s + 1] - f;
        const int32_t *rows = S->rows + S->rowptr[s];
        const double *P = L->Lx + L->lxptr[s];
        blas_int bc = c, br = (blas_int)r, bm = (blas_int)(r - c);
        BLASNAME(dtrsv)("L", "N", "N", &bc, P, &br, y + f, &inc);
        if (bm > 0) {
            BLASNAME(dgemv)("N", &bm, &bc, &one, P + c, &br, y + f, &inc, &zero, tmp, &inc);
            for (int64_t t = 0; t < r - c; t++) y[rows[c + t]] -= tmp[t];
        }
    }
    for (int32_t s = S->nsuper - 1; s >= 0; s--) {      /* backward: L^T z = y */
        const int64_t r = S->rowptr[s + 1] - S->rowptr[s];
        const int32_t f = S->sfirst[s], c = S->sfirst[s + 1] - f;
        const int32_t *rows = S->rows + S->rowptr[s];
        const double *P = L->Lx + L->lxptr[s];
        blas_int bc = c, br = (blas_int)r, bm = (blas_int)(r - c);
        if (bm > 0) {
            const double mone = -1.0;
            for (int64_t t = 0; t < r - c; t++) tmp[t] = y[rows[c + t]];
            BLASNAME(dgemv)("T", &bm, &bc, &mone, P + c, &br, tmp, &inc, &one, y + f, &inc);
        }
        BLASNAME(dtrsv)("L", "T", "N", &bc, P, &br, y + f, &inc);
    }
    for (int64_t i = 0; i < n; i++) x[S->perm[i]] = y[i];
    cc->status = CHOLMOD_OK;
    return 1;
}

int cholmod_l_free_factor(cholmod_factor **L, cholmod_common *cc) {
    (void)cc;
    if (!L || !*L) return 1;
    cholmod_factor *F = *L;
    spx_symbolic_free(&F->S);
    free(F->rp); free(F->ci); free(F->cx); free(F->lxptr); free(F->Lx);
    free(F);
    *L = NULL;
    return 1;
}

int cholmod_l_free_dense(cholmod_dense **X, cholmod_common *cc) {
    (void)cc;
    if (!X || !*X) return 1;
    free((*X)->x);
    free(*X);
    *X = NULL;
    return 1;
}
