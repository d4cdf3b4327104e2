/* speigs.h -- C ABI of the B200 sparse symmetric eigensolver.
 *
 * Drop-in for the reference interface include/speigs.h (moatas19m/sparse-eigs-mex):
 * the same type names, enum values, struct layouts and function signatures,
 * so a caller compiled against the reference header links against
 * libspeigs.so unchanged.  Each declaration below names the reference line
 * it replaces.
 *
 * Only the 'sm' (shift-invert Lanczos through a supernodal Cholesky) and
 * 'lm' (direct Lanczos) hot paths run their numerical work on the GPU; the
 * structure checks, component split and symbolic analysis stay on the host.
 */
#ifndef SPEIGS_H
#define SPEIGS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Index type of the CSC arrays (reference include/speigs.h:21). */
typedef int64_t speigs_int;

/* Which end of the spectrum (reference include/speigs.h:23-26). */
typedef enum {
    SPEIGS_SM = 0,   /* k smallest in magnitude: shift-invert Lanczos */
    SPEIGS_LM = 1    /* k largest in magnitude: Lanczos on A itself   */
} speigs_which;

/* Route taken by the structure analysis (reference include/speigs.h:30-38). */
typedef enum {
    SPEIGS_PATH_DIAG      = 0,  /* diagonal matrix                         */
    SPEIGS_PATH_DENSE     = 1,  /* small n or large k/n: dense eigensolver */
    SPEIGS_PATH_SHIFTINV  = 2,  /* Cholesky shift-invert Lanczos           */
    SPEIGS_PATH_DIRECT    = 3,  /* Lanczos on A ('lm')                     */
    SPEIGS_PATH_BLOCKS    = 4,  /* solved per connected component          */
    SPEIGS_PATH_LU        = 5,  /* indefinite: LU shift-invert             */
    SPEIGS_PATH_BANDED    = 6   /* narrow band after RCM                   */
} speigs_path;

/* Options; a zero field selects the default (reference include/speigs.h:40-55). */
typedef struct {
    double      tol;        /* ||Av - lv|| <= tol*max(||A||_1,1); 0 => 1e-14   */
    speigs_int  maxit;      /* restarts; 0 => 300                              */
    speigs_int  ncv;        /* Krylov basis size; 0 => max(2k+1, 20)           */
    int         dense_max;  /* dense route when n <= this; -1 => 800, 0 => off */
    int         detect;     /* 1 => structure analysis (default), 0 => off     */
    uint64_t    seed;       /* start-vector seed; 0 => 88172645463325252       */
    int         check_sym;  /* 1 => reject non-symmetric input (default)       */
    int         band_max;   /* banded route when RCM bandwidth <= this         */
    int         ordering;   /* 0 auto, 1 minimum degree, 2 nested dissection   */
    double      shift0;     /* first delta for a singular A, relative to ||A||_1 */
} speigs_opts;

/* Diagnostics (reference include/speigs.h:57-68). */
typedef struct {
    int         flag;       /* 0 = all k converged, 1 = partial                */
    speigs_int  nconv;
    speigs_int  restarts;
    speigs_int  nops;       /* operator applications (solves or products)     */
    double      shift;      /* delta used in A + delta*I                       */
    double      anorm;      /* ||A||_1                                         */
    speigs_path path;
    speigs_int  ncomp;      /* connected components (1 if not split)           */
    double      t_analyze, t_factor, t_iter;
    double      t_op, t_ortho, t_resid, t_ritz;
} speigs_info;

/* Fill *o with defaults (reference include/speigs.h:70). */
void speigs_default_opts(speigs_opts *o);

/* k eigenpairs of the n x n symmetric matrix given in CSC (full or upper
 * storage, rows sorted within a column; only the upper triangle is read).
 * lambda[k] out (required), V[n*k] column-major out (may be NULL),
 * resid[k] out (may be NULL).  Returns 0 or a negative SPEIGS_ERR_* code.
 * (reference include/speigs.h:81-84) */
int speigs(speigs_int n,
           const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
           speigs_int k, speigs_which which, const speigs_opts *opts,
           double *lambda, double *V, double *resid, speigs_info *info);

/* Complex Hermitian A = Axr + i*Axi through its real 2n x 2n embedding.
 * Axi == NULL is the real case.  (reference include/speigs.h:92-97) */
int speigs_z(speigs_int n,
             const speigs_int *Ap, const speigs_int *Ai,
             const double *Axr, const double *Axi,
             speigs_int k, speigs_which which, const speigs_opts *opts,
             double *lambda, double *Vr, double *Vi, double *resid,
             speigs_info *info);

/* Text for a return code (reference include/speigs.h:99). */
const char *speigs_errmsg(int code);

/* Return codes (reference include/speigs.h:101-107). */
#define SPEIGS_OK             0
#define SPEIGS_ERR_ARG      (-1)
#define SPEIGS_ERR_MEM      (-2)
#define SPEIGS_ERR_FACTOR   (-3)
#define SPEIGS_ERR_LAPACK   (-4)
#define SPEIGS_ERR_INTERNAL (-5)
#define SPEIGS_ERR_NOTSYM   (-6)

#ifdef __cplusplus
}
#endif
#endif /* SPEIGS_H */
