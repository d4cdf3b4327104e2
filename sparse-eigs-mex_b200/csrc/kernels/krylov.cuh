// Launch wrappers of the Krylov-side kernels (SpMV, tall-skinny Gram-Schmidt,
// Ritz vectors and residuals, start vectors, the projected eigenproblem).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spx {

// Reduction scratch shared by the tall-skinny kernels: per-block partial
// sums plus a completion counter (the last block to finish reduces).
struct ReduceScratch {
    double   *part    = nullptr;  // capacity: max_blocks * max_cols doubles
    unsigned *counter = nullptr;  // one counter, zero between launches
    int       max_blocks = 0;
    int       max_cols   = 0;
};

// y = A x for the full symmetric CSR (int32 row pointers and columns).
void launch_spmv(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                 const double *x, double *y, cudaStream_t st);

// Tall-skinny Gram-Schmidt passes over V (n x m, column-major, ld = ldv).
//   dot:         h = V^T w
//   update_dot:  w -= V hin, then h = V^T w
//   update_norm: w -= V hin, then nrm2 = w^T w
//   norm:        nrm2 = w^T w
// hcol (optional): the projected-matrix column; hmode 1 assigns h, 2 adds h.
void launch_ts_dot(const double *V, int64_t ldv, int n, int m, const double *w, double *h,
                   double *hcol, int hmode, const ReduceScratch &rs, cudaStream_t st);
void launch_ts_update_dot(const double *V, int64_t ldv, int n, int m, double *w,
                          const double *hin, double *h, double *hcol, int hmode,
                          const ReduceScratch &rs, cudaStream_t st);
void launch_ts_update_norm(const double *V, int64_t ldv, int n, int m, double *w,
                           const double *hin, double *nrm2, const ReduceScratch &rs,
                           cudaStream_t st);
void launch_ts_norm(int n, const double *w, double *nrm2, const ReduceScratch &rs,
                    cudaStream_t st);

// dst = src * (1 / sqrt(nrm2[0]))   (the reciprocal is formed first, as dscal does)
void launch_scale_by_invnorm(int n, const double *src, const double *nrm2, double *dst,
                             cudaStream_t st);

// X[:, t] = V[:, 0:m] * S[:, idx[t]]  for t < nvec; nrm2[t] = ||X[:, t]||^2
void launch_ritz_vectors(const double *V, int64_t ldv, int n, int m, const double *S, int lds,
                         const int *idx, int idx_off, int nvec, double *X, int64_t ldx,
                         double *nrm2, const ReduceScratch &rs, cudaStream_t st);
// X[:, t] *= 1/sqrt(nrm2[t]) where nrm2[t] > 0
void launch_scale_cols(int n, int nvec, double *X, int64_t ldx, const double *nrm2,
                       cudaStream_t st);
// lam[t] = x_t . Ax_t ; then r2[t] = ||Ax_t - lam_t x_t||^2
void launch_rayleigh_resid(int n, int nvec, const double *X, int64_t ldx, const double *AX,
                           int64_t ldax, double *lam, double *r2, const ReduceScratch &rs,
                           cudaStream_t st);

// Start vector: v[i] = uniform [-0.5, 0.5) from the xorshift64* stream whose
// state is `seed`, advanced i+1 times (bit-identical to a sequential draw).
void launch_rand_vec(int n, uint64_t seed, double *v, cudaStream_t st);
// State after `steps` draws (host, exact jump-ahead).
uint64_t rng_advance(uint64_t seed, uint64_t steps);
// The jump table behind it (host, 64 x 64 words: entry [b][j] is M^(2^b) e_j
// for the xorshift64* state update M), for kernels that jump on the device.
const uint64_t *rng_jump_table();

// Projected eigenproblem: symmetric m x m matrix H (column-major, ld = ldh)
// -> theta[m] ascending, eigenvectors S (m x m, ld = m), and ord[m]: the
// indices sorted by |theta| descending (stable).  One thread block.
// work: >= 2*m_even^2 doubles of global workspace for m too large for
// shared memory.  status[0] gets the sweep count (negative if not converged).
void launch_syev_small(int m, const double *H, int ldh, double *theta, double *S, int *ord,
                       double *work, int *status, cudaStream_t st);
int syev_small_smem_limit();
// The same eigensolver on nprob problems at once, one block each: problem b
// has order mvec[b] (or m when mvec is null; every order <= m <=
// syev_small_smem_limit()), reads H + b * strideH (leading dimension ldh)
// and writes theta[b*m ..], S[b*m*m ..] (ld its order), ord[b*m ..] and
// status[2b]; problems with active[b] == 0 are skipped (active may be null).
void launch_syev_batched(int nprob, int m, const int *mvec, const double *H, int ldh,
                         int64_t strideH, double *theta, double *S, int *ord, int *status,
                         const int *active, cudaStream_t st);
// Same eigensolver, always keeping its two m x m matrices in the caller's
// global workspace `work` (>= 2*m_even^2 doubles); shared memory holds only
// the rotation parameters.
void launch_syev_small_workspace(int m, const double *H, int ldh, double *theta, double *S,
                                 int *ord, double *work, int *status, cudaStream_t st);

// H (ldh x ldh) = diag(d[0..nd)) with zeros elsewhere in the leading m x m part
void launch_set_diag(int ldh, int nd, const double *d, double *H, cudaStream_t st);
// H[r + c*ldh] = H[c + r*ldh] = sqrt(nrm2[0]) or 0 if zero_flag
// *flag = 1 when nrm2[0] < thr (device-side test of a squared norm)
void launch_flag_if_below(const double *nrm2, double thr, int *flag, cudaStream_t st);
void launch_set_beta(double *H, int ldh, int r, int c, const double *nrm2, int zero,
                     cudaStream_t st);

// Iterative refinement of a solve with a lower-precision factor:
//   r = b - (A + shift I) y, and flag <- 1 once
//   ||r|| <= tol * (anorm ||y|| + ||b||)   (a backward-error test);
// while the flag is 0 every evaluation adds one to *count (a correction
// follows).  Does nothing when *flag is already set.
void launch_refine_residual(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                            double shift, const double *b, const double *y, double *r,
                            double tol, double anorm, int *flag, int *count,
                            const ReduceScratch &rs, cudaStream_t st);
// y += d unless *flag
void launch_axpy_unless(int n, double *y, const double *d, const int *flag, cudaStream_t st);

// y = a x + b y
void launch_axpby(int64_t n, double a, const double *x, double b, double *y, cudaStream_t st);

// generic helpers
void launch_copy(int64_t n, const double *src, double *dst, cudaStream_t st);
void launch_fill(int64_t n, double v, double *dst, cudaStream_t st);

}  // namespace spx
