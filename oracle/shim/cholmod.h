/* ORACLE TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * A project-written stand-in for the subset of SuiteSparse CHOLMOD (v7.14.0,
 * the version the reference pins in build_suitesparse.sh:16) that the
 * reference's src/speigs_core.c uses, so that file compiles UNMODIFIED from
 * the reference tree and runs here as the CPU oracle and CPU baseline.
 * Identifiers, field names and constant names follow CHOLMOD's published
 * interface because the reference source names them; the implementation
 * behind them (cholmod_shim.c) is this project's own: a CPU multifrontal
 * supernodal LL^T over BLAS-3, on the host nested-dissection ordering.
 */
#ifndef ORACLE_CHOLMOD_SHIM_H
#define ORACLE_CHOLMOD_SHIM_H
#include <stddef.h>
#include <stdint.h>

#define CHOLMOD_OK          0
#define CHOLMOD_NOT_POSDEF  1
#define CHOLMOD_SIMPLICIAL  0
#define CHOLMOD_AUTO        1
#define CHOLMOD_SUPERNODAL  2
#define CHOLMOD_NATURAL     0
#define CHOLMOD_GIVEN       1
#define CHOLMOD_AMD         2
#define CHOLMOD_METIS       3
#define CHOLMOD_INT         0
#define CHOLMOD_LONG        2
#define CHOLMOD_PATTERN     0
#define CHOLMOD_REAL        1
#define CHOLMOD_DOUBLE      0
#define CHOLMOD_A           0
#define CHOLMOD_MAXMETHODS  9

typedef struct cholmod_method_struct { int ordering; } cholmod_method_struct;

typedef struct cholmod_common {
    int    supernodal;
    int    print;
    void (*error_handler)(int status, const char *file, int line, const char *msg);
    int    nmethods;
    int    postorder;
    cholmod_method_struct method[CHOLMOD_MAXMETHODS + 1];
    int    status;
    int    nthreads;
} cholmod_common;

typedef struct cholmod_sparse {
    size_t nrow, ncol, nzmax;
    void  *p, *i, *nz, *x, *z;
    int    stype, itype, xtype, dtype, sorted, packed;
} cholmod_sparse;

typedef struct cholmod_dense {
    size_t nrow, ncol, nzmax, d;
    void  *x, *z;
    int    xtype, dtype;
} cholmod_dense;

typedef struct cholmod_factor cholmod_factor;   /* opaque */

int    cholmod_l_start(cholmod_common *cc);
int    cholmod_l_finish(cholmod_common *cc);
double cholmod_l_norm_sparse(cholmod_sparse *A, int norm, cholmod_common *cc);
int    cholmod_l_sdmult(cholmod_sparse *A, int transpose, double alpha[2], double beta[2],
                        cholmod_dense *X, cholmod_dense *Y, cholmod_common *cc);
cholmod_factor *cholmod_l_analyze(cholmod_sparse *A, cholmod_common *cc);
int    cholmod_l_factorize_p(cholmod_sparse *A, double beta[2], int64_t *fset, size_t fsize,
                             cholmod_factor *L, cholmod_common *cc);
int    cholmod_l_solve2(int sys, cholmod_factor *L, cholmod_dense *B, cholmod_sparse *Bset,
                        cholmod_dense **X_Handle, cholmod_sparse **Xset_Handle,
                        cholmod_dense **Y_Handle, cholmod_dense **E_Handle, cholmod_common *cc);
int    cholmod_l_free_factor(cholmod_factor **L, cholmod_common *cc);
int    cholmod_l_free_dense(cholmod_dense **X, cholmod_common *cc);
#endif
