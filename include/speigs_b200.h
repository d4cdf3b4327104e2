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

/* ---- extension options: precision of the shift-invert operator ------------
 * SPEIGS_B200_FP64: the drop-in path, an FP64 supernodal factor.
 * SPEIGS_B200_MIXED ('sm' only): the factor is stored in FP32 and its
 * trailing updates run on the TF32 tensor cores with an FP32-accurate
 * three-term split; every solve is refined in FP64 (r = b - (A+dI)y,
 * y += M^{-1} r) until ||r|| <= refine_tol * (||A||_1 ||y|| + ||b||) or
 * refine_max corrections were made.  The Lanczos recurrence, the
 * reorthogonalisation, the Ritz problem and the residuals stay FP64.
 * No counterpart in the reference interface. */
#define SPEIGS_B200_FP64  0
#define SPEIGS_B200_MIXED 1

typedef struct {
    int          precision;    /* SPEIGS_B200_FP64 (default) or SPEIGS_B200_MIXED     */
    int          refine_max;   /* corrections per solve (mixed); 0 => 10               */
    double       refine_tol;   /* backward-error target (mixed); 0 => 1e-2 tol, within
                                  [1e-14, 1e-12]                                        */
    const double *warm;        /* optional start subspace, n x warm_cols, column-major,
                                  host or device memory (on the calling thread's
                                  device); NULL => the reference's random start       */
    speigs_int   warm_cols;
    int          block;        /* 'sm' Krylov method (see below); 0 => automatic        */
    int          handoff;      /* speigs_batched: the lockstep loop hands its components
                                  still iterating to the per-component executor once they
                                  hold at most 1/handoff of the rows; 0 => 8, -1 => never */
} speigs_ext_opts;

/* speigs_ext_opts.block selects the Krylov method of the 'sm' route:
 *   0   automatic: with a start subspace (warm), a block thick-restart
 *       Lanczos whose first block is that subspace (width min(warm_cols,
 *       32)); without one, the reference's single-vector Lanczos;
 *   b   (1..32) the block method with blocks of b vectors; a start subspace
 *       fills the first block, the reference's random stream the rest;
 *  -1   the single-vector Lanczos always; a start subspace is then folded
 *       into its start vector.
 * The block method reads the factor once per block of b vectors (one
 * persistent launch for all of them) and converges to the same eigenpairs
 * under the same test: ||A x - lambda x|| <= tol max(||A||_1, 1) for the k
 * wanted pairs.  Its operator-application count (speigs_info.nops) counts
 * vectors; its restart count counts restart cycles. */

typedef struct {
    int          precision;      /* precision actually used                         */
    speigs_int   refine_steps;   /* FP64 refinement corrections made (mixed)        */
    speigs_int   factor_solves;  /* solves with the factor: applications + corrections */
    speigs_int   warm_cols;      /* start-subspace columns used (0: random start)   */
    int          block;          /* block size of the block method (0: single vector) */
    speigs_int   block_solves;   /* block solves: applications + corrections        */
    /* host wall time (s) of the Krylov route outside speigs_info's t_analyze /
     * t_factor / t_iter: input checks and the CSR build, plan set-up (device
     * buffers, uploads), copy-out and release */
    double       t_checks, t_setup, t_release;
    /* block method: device time (s) of the block solves (their layout
     * conversions included) and the number queued, corrections that returned
     * at once on the device included */
    double       t_block_solve;
    speigs_int   block_solve_calls;
} speigs_ext_info;

/* Fill *e with the defaults (FP64, no start subspace). */
void speigs_default_ext_opts(speigs_ext_opts *e);

/* speigs() with extension options; ext == NULL is speigs() itself.  einfo
 * (may be NULL) receives the extension diagnostics of the Krylov route. */
int speigs_ex(speigs_int n, const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
              speigs_int k, speigs_which which, const speigs_opts *opts,
              const speigs_ext_opts *ext, double *lambda, double *V, double *resid,
              speigs_info *info, speigs_ext_info *einfo);

/* ---- batched components --------------------------------------------------
 * speigs() splits a matrix into its connected components, solves each and
 * keeps the global k of the merged candidates (reference blocks_path,
 * src/speigs_core.c:532-632).  These two calls keep k eigenpairs of EVERY
 * component instead.  The components are solved concurrently (a host
 * thread pool, every solve on its own CUDA stream).  No counterpart in the
 * reference interface. */

/* Connected components over the numerically nonzero entries of the upper
 * triangle, labelled in order of first appearance -- the split speigs()
 * makes.  comp[n] receives the labels, *ncomp their count. */
int speigs_components(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                      const double *Ax, speigs_int *comp, speigs_int *ncomp);

/* min(k, n_c) eigenpairs of every component c (labels from
 * speigs_components).  lambda[ncomp*k]: row c (entries c*k .. c*k+k-1)
 * holds component c's values sorted as speigs() sorts them, zero-filled;
 * V[n*k] (may be NULL): column t holds the t-th eigenvector of every
 * component on that component's rows; resid[ncomp*k] (may be NULL);
 * nvals[ncomp] (may be NULL) receives min(k, n_c).  info (may be NULL):
 * operator applications summed, flag = 1 if any component is partial,
 * ncomp, path = SPEIGS_PATH_BLOCKS.  ext may be NULL. */
int speigs_batched(speigs_int n, const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
                   speigs_int k, speigs_which which, const speigs_opts *opts,
                   const speigs_ext_opts *ext, const speigs_int *comp, speigs_int ncomp,
                   double *lambda, double *V, double *resid, speigs_int *nvals,
                   speigs_info *info);

/* Phases of the calling thread's last speigs_batched call.  No counterpart in
 * the reference interface.  times[9] (seconds): input checks and the
 * component split; building the lockstep group's CSR; the group's symbolic
 * analysis, numeric factorization and Lanczos iterations; the lockstep part
 * in all; the components solved one by one (dense gate, singular forests,
 * extension options, stragglers handed off); the whole call; the lockstep
 * engine's own total.  counts[7]: components in the lockstep group,
 * components solved one by one, stragglers handed off, lockstep steps,
 * restart cycles, rows of the lockstep group, 1 if its step ran as a CUDA
 * graph. */
int speigs_b200_batched_stats(double *times, int64_t *counts);

/* ---- learned warm start: the message-passing network -----------------------
 * h0 = tanh(W0 x + b0); h_l = tanh(W_l [h_{l-1}, A h_{l-1}] + b_l), l = 1..L;
 * Y = W_o h_L + b_o.  x: nfeat features per node (FP32), A: a sparse
 * normalised adjacency given as CSR (int32 row pointers and columns, FP32
 * weights), Y: nout channels per node (FP32), all row-major (node-major) and
 * in DEVICE memory.  Weights and activations are BF16 with FP32
 * accumulation; the optimiser (Adam) keeps FP32 weights.  Training
 * minimises 1 - trace(U^T P_Y U) / k, the share of the k target vectors U
 * (orthonormal columns, node-major n x k) outside span(Y).  hidden must be
 * 64; nfeat, nout <= 64; layers <= 8.  Calls on one network must not overlap.
 * No counterpart in the reference interface. */
typedef struct speigs_mpnn_s *speigs_mpnn;
int  speigs_b200_mpnn_create(int nfeat, int hidden, int layers, int nout, uint64_t seed,
                             speigs_mpnn *net);
void speigs_b200_mpnn_destroy(speigs_mpnn net);
/* Kernels of the forward pass's dense layers: on = 1 (the default) runs the
 * BF16 layers whose shapes fit (inputs 16..128 wide in multiples of 16,
 * at most 64 outputs, 16-byte aligned rows) on the tensor cores (tcgen05,
 * FP32 accumulation in TMEM), on = 0 runs every layer on the FP32-FMA
 * kernels; on < 0 only queries.  Returns the previous setting, or
 * SPEIGS_ERR_ARG for a null network.  The two differ only in the order of
 * the FP32 sums. */
int  speigs_b200_mpnn_tensor_cores(speigs_mpnn net, int on);
/* The network's input graph for an N x N x N finite-volume grid, built on
 * the device: the normalised adjacency w_ij = t_ij / sqrt(s_i s_j) of the
 * operator with face transmissibilities t = 2 k_a k_b / (k_a + k_b) from the
 * cell conductivities kap (N^3 doubles, index (a0 N + a1) N + a2), s_i the
 * sum of node i's t.  Rows in node order, neighbours ascending; rowptr has
 * N^3 + 1 entries, col and w room for 6 N^2 (N - 1).  All pointers are
 * device memory; queued on `stream`.  Returns 0 or a negative code. */
int  speigs_b200_mpnn_grid_graph(speigs_mpnn net, int N, const double *kap, int32_t *rowptr,
                                 int32_t *col, float *w, void *stream);
/* FP32 weights to (set = 0) or from (set = 1) host memory; host == NULL
 * reports the count in *count. */
int  speigs_b200_mpnn_params(speigs_mpnn net, float *host, int64_t *count, int set);
/* Gradient of the last training step (FP32, host). */
int  speigs_b200_mpnn_grads(speigs_mpnn net, float *host);
int  speigs_b200_mpnn_forward(speigs_mpnn net, int64_t n, const int32_t *rowptr,
                              const int32_t *col, const float *w, const float *X, float *Y,
                              void *stream);
/* Forward, loss, backward and (lr > 0) one Adam step; *loss receives the
 * loss before the step. */
int  speigs_b200_mpnn_train_step(speigs_mpnn net, int64_t n, const int32_t *rowptr,
                                 const int32_t *col, const float *w, const float *X,
                                 const float *U, int k, float lr, double *loss, void *stream);

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

/* speigs_plan_create with extension options (precision; the start subspace
 * is taken per solve from ext->warm when given here). */
int speigs_plan_create_ex(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                          const double *Ax, speigs_which which, const speigs_opts *opts,
                          const speigs_ext_opts *ext, speigs_plan *plan);

/* Extension diagnostics of the plan's last solve. */
int speigs_plan_ext_info(speigs_plan plan, speigs_ext_info *einfo);

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

/* Y = Op X for nr <= 32 vectors at once (X, Y column-major n x nr device
 * arrays, leading dimensions ldx, ldy >= n).  For 'sm' one persistent launch
 * solves all nr columns, reading the factor once (mixed precision: each
 * column refined in FP64 as in speigs_plan_apply_device); for 'lm' the
 * columns are multiplied by A one after another.  No counterpart in the
 * reference interface. */
int speigs_plan_apply_block_device(speigs_plan plan, const double *X, int64_t ldx, double *Y,
                                   int64_t ldy, int nr);

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

/* The same contract on a host core: Householder tridiagonalisation and the
 * implicit symmetric QR iteration with Wilkinson shifts.  H has leading
 * dimension ldh >= m; all buffers are host memory.  This is the solver the
 * Lanczos loops of speigs() use for their projected problem (the reference
 * calls LAPACK dsyev on the host there, src/speigs_core.c:180, :236).
 * Returns 0, or -1 for bad arguments or when the iteration did not converge
 * within 30 m steps. */
int speigs_b200_syev_small_host(int m, const double *H, int ldh, double *theta, double *S,
                                int *ord);

/* The same contract with eigenvectors for the nvec leading entries of ord
 * only (the other columns of S are set to zero): Householder reduction of
 * the lower triangle, the implicit QR on the eigenvalues alone (theta agrees
 * with speigs_b200_syev_small_host's to rounding), inverse iteration on the
 * tridiagonal with
 * Gram-Schmidt inside clusters of close eigenvalues, and the reflectors
 * applied to the vectors -- LAPACK dsyevx's method, O(m^2) per vector.  The
 * block Lanczos method solves its projected problem with it (its restart
 * and residual test read only the wanted Ritz vectors).  nvec >= m solves
 * fully.  Returns 0, or -1 for bad arguments or no convergence. */
int speigs_b200_syev_select_host(int m, const double *H, int ldh, int nvec, double *theta,
                                 double *S, int *ord);

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
 * array's device address; make that first call before any stream capture.
 * That address is kept per device ordinal for the life of the process, so it
 * belongs to the context that was current at the first call: after
 * cudaDeviceReset, or with a different driver context made current on that
 * device, do not call this entry point again.  If a CUDA error from earlier
 * work is pending on the calling thread, nothing is launched and the call
 * returns SPEIGS_ERR_INTERNAL, naming that error. */
int speigs_b200_syev_small_noalloc(int m, const double *H, double *theta, double *S, int *ord,
                                   int *status, void *stream);

/* Factorization cache of speigs() / speigs_ex() (opt-in; off by default).
 * With entries > 0 the device-resident plans -- the matrix, its symbolic
 * analysis and its numeric factor -- of the last `entries` distinct
 * operators that reached the Krylov route are kept, keyed by the matrix's
 * contents (the symmetric matrix of its upper triangle, compared in full),
 * the route, the factor options (ordering, shift0), the precision and the
 * current device.  A later call on the same operator skips the analysis and
 * the factorization (speigs_info t_analyze is then 0 and t_factor ~0); the
 * Lanczos options (k, tol, ncv, maxit, seed) may differ between calls.  The
 * kept plans hold device memory until they are evicted (least recently used
 * first) or the cache is resized; entries = 0 releases them all.  Calls on
 * other threads that want an entry in use build their own plan.  The
 * reference documents this cache as a planned feature (docs/REQUIREMENTS.md);
 * its speigs.h has no counterpart.  Returns SPEIGS_OK or SPEIGS_ERR_ARG. */
int speigs_b200_factor_cache(int entries);
/* Plans currently kept by the factorization cache. */
int speigs_b200_factor_cache_size(void);

/* Process-wide counts since the library was loaded: kernels this library
 * launched, and bytes it copied host->device and device->host. */
void speigs_b200_counters(long long *launches, long long *h2d_bytes, long long *d2h_bytes);

/* Text of the last CUDA failure seen on this thread ("" if none). */
const char *speigs_b200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SPEIGS_B200_H */
