/* speigs_b200.h -- extension entry points of the B200 library.
 *
 * Nothing here replaces a reference symbol: these entry points have no
 * counterpart in the reference interface (include/speigs.h of
 * moatas19m/sparse-eigs-mex).  They let a caller keep a matrix resident on
 * the GPU between solves (a family of operators with one sparsity pattern,
 * or repeated solves while benchmarking) and expose the operator and the
 * building blocks for testing.  The plain drop-in is speigs.h alone.
 */
#ifndef SPEIGS_B200_H
#define SPEIGS_B200_H

#include <stddef.h>
#include "speigs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque solver plan: one connected symmetric matrix on one GPU, with its
 * operator ('sm': symbolic analysis done, numeric factor per solve; 'lm':
 * the matrix itself) and every device buffer the Lanczos iteration needs.
 * A plan owns a CUDA stream; calls on one plan must not overlap. */
typedef struct speigs_plan_s *speigs_plan;

/* Host set-up of the 'sm'/'lm' route for a matrix that speigs() would send
 * to the Krylov path (no diagonal, dense or component split is attempted):
 * symmetry check (when opts->check_sym), ||A||_1, the full CSR, the ordering
 * and symbolic analysis, and the copy of the matrix to the GPU.
 * Returns SPEIGS_OK or a negative code. */
int speigs_plan_create(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                       const double *Ax, speigs_which which, const speigs_opts *opts,
                       speigs_plan *plan);

/* New values for the same pattern.  Ax follows the CSC given at creation
 * (host pointer); only the upper triangle is read. */
int speigs_plan_set_values(speigs_plan plan, const double *Ax);

/* Numeric factorization ('sm', with the capped shift escalation) and the
 * thick-restart Lanczos, with the k results written to DEVICE memory:
 * lambda[k], V[n*k] column-major (may be NULL), resid[k] (may be NULL),
 * sorted by |lambda| as speigs() sorts them.  info may be NULL. */
int speigs_plan_solve_device(speigs_plan plan, speigs_int k, double *lambda, double *V,
                             double *resid, speigs_info *info);

/* y = Op x on the device (Op = A for 'lm', (A + shift I)^{-1} for 'sm' after
 * a solve or speigs_plan_factor); x, y are device vectors of length n. */
int speigs_plan_apply_device(speigs_plan plan, const double *x, double *y);

/* Numeric factorization only ('sm'); *shift receives the delta used. */
int speigs_plan_factor(speigs_plan plan, double *shift);

/* The CUDA stream the plan runs on (a cudaStream_t), so a caller can order
 * its own work or events against the plan's. */
void *speigs_plan_stream(speigs_plan plan);

/* Algorithmic traffic/work figures of the plan's operator: bytes of one
 * operator application and flops of one numeric factorization. */
int speigs_plan_costs(speigs_plan plan, double *op_bytes, double *factor_flops,
                      double *nnz_factor);

void speigs_plan_destroy(speigs_plan plan);

/* Device start vector: v[0..n) (host buffer) drawn on the GPU from the
 * xorshift64* stream used by the reference (src/speigs_core.c:49-54). */
int speigs_b200_rand_vec(speigs_int n, uint64_t seed, double *v);

/* Projected eigenproblem on the GPU (one thread block): H is m x m
 * column-major (host), only its upper triangle is read.  theta[m]
 * ascending, S[m*m] eigenvectors, ord[m] indices by |theta| descending. */
int speigs_b200_syev_small(int m, const double *H, double *theta, double *S, int *ord);

/* Allocation-free variant of speigs_b200_syev_small.  No counterpart in the
 * reference interface.  For callers that cannot call cudaMalloc where they
 * need the solve -- code running under CUDA stream capture, real-time loops
 * that must not touch the allocator, hosts whose device memory belongs to
 * another allocator.  All pointers are DEVICE memory owned by the caller: H
 * (m x m column-major, upper triangle read), theta[m], S[m*m], ord[m];
 * status (optional, may be NULL) receives the sweep count, negative if the
 * sweeps did not converge.  The work is enqueued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream) and the call returns
 * without waiting.  m must be 1..256: larger sizes return SPEIGS_ERR_ARG.
 * The workspace is a 1 MiB array compiled into the library, held by every
 * GPU that loads it until the process exits and shared by all calls: calls
 * that overlap on the GPU race.  The first call on each device looks up the
 * array's device address; make that first call before any stream capture. */
int speigs_b200_syev_small_noalloc(int m, const double *H, double *theta, double *S, int *ord,
                                   int *status, void *stream);

/* Process-wide counts since the library was loaded: kernels this library
 * launched, and bytes it copied host->device and device->host. */
void speigs_b200_counters(long long *launches, long long *h2d_bytes, long long *d2h_bytes);

/* Text of the last CUDA failure seen on this thread ("" if none). */
const char *speigs_b200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SPEIGS_B200_H */
