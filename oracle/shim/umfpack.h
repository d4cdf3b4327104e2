/* ORACLE TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * Project-written stand-in for the UMFPACK (SuiteSparse v7.14.0) entry points
 * that the reference's src/speigs_core.c (:111-115, :979-983) and
 * bench/bench_model.c use.  Names follow UMFPACK's published interface; the
 * implementation (umfpack_shim.c) is a dense LU with partial pivoting from
 * LAPACK, sized for the reference's indefinite-fallback test cases only.
 */
#ifndef ORACLE_UMFPACK_SHIM_H
#define ORACLE_UMFPACK_SHIM_H
#include <stdint.h>

#define UMFPACK_CONTROL 20
#define UMFPACK_INFO    90
#define UMFPACK_A        0
#define UMFPACK_OK       0
#define UMFPACK_WARNING_singular_matrix      1
#define UMFPACK_ERROR_out_of_memory        (-1)
#define UMFPACK_ERROR_invalid_matrix       (-8)

void umfpack_dl_defaults(double Control[UMFPACK_CONTROL]);
int  umfpack_dl_symbolic(int64_t n_row, int64_t n_col, const int64_t *Ap, const int64_t *Ai,
                         const double *Ax, void **Symbolic, const double *Control, double *Info);
int  umfpack_dl_numeric(const int64_t *Ap, const int64_t *Ai, const double *Ax, void *Symbolic,
                        void **Numeric, const double *Control, double *Info);
int  umfpack_dl_solve(int sys, const int64_t *Ap, const int64_t *Ai, const double *Ax, double *X,
                      const double *B, void *Numeric, const double *Control, double *Info);
void umfpack_dl_free_symbolic(void **Symbolic);
void umfpack_dl_free_numeric(void **Numeric);
#endif
