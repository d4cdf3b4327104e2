// Launch wrappers of the block Krylov kernels: the tall-skinny products of a
// block thick-restart Lanczos (a block of b <= 32 vectors against a basis of
// m <= 128 vectors), the Cholesky QR of a block, and the FP64 refinement
// residual of a block solve.  Every array is column-major with an explicit
// leading dimension.  Sums are formed in a fixed order, so results repeat
// bit for bit from run to run.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spx {

constexpr int kBlockMaxB = 32;    // vectors per block
constexpr int kBlockMaxM = 128;   // basis vectors a block is projected against

// Partial sums of the tall-skinny products: per row-range block, m x b
// doubles, then reduced across the row ranges in a second launch.
struct BlockScratch {
    double *part = nullptr;       // capacity: max_parts * kBlockMaxM * kBlockMaxB doubles
    int     max_parts = 0;
};
// Row-range blocks a product over n rows uses (<= 2 per SM).
int tsb_parts(int n);

// H[0:m, 0:b] = V[:, 0:m]^T W[:, 0:b]  (mode 0), or += (mode 1).
void launch_tsb_tn(const double *V, int64_t ldv, int n, int m, const double *W, int64_t ldw,
                   int b, double *H, int ldh, int mode, const BlockScratch &bs, cudaStream_t st);
// W[:, 0:b] -= V[:, 0:m] H[0:m, 0:b]
void launch_tsb_nn_sub(const double *V, int64_t ldv, int n, int m, const double *H, int ldh,
                       double *W, int64_t ldw, int b, cudaStream_t st);
// W[:, 0:b] -= V[:, 0:m] H1, then H2[0:m, 0:b] = V^T W (mode 0) or += (mode
// 1), in one sweep over V; the results equal, bit for bit, those of
// launch_tsb_nn_sub followed by launch_tsb_tn.  H2 may be H1.
void launch_tsb_sub_tn(const double *V, int64_t ldv, int n, int m, const double *H1, int ldh1,
                       double *W, int64_t ldw, int b, double *H2, int ldh2, int mode,
                       const BlockScratch &bs, cudaStream_t st);
// W[:, 0:b] -= V[:, 0:m] H1, then G = W^T W (b x b, leading dimension b),
// in one sweep; bit for bit launch_tsb_nn_sub followed by launch_tsb_tn(W, W).
void launch_tsb_sub_gram(const double *V, int64_t ldv, int n, int m, const double *H1, int ldh1,
                         double *W, int64_t ldw, int b, double *G, const BlockScratch &bs,
                         cudaStream_t st);
// W[:, 0:b] = W Rinv (Rinv b x b, leading dimension b), then G = W^T W, in one
// sweep; bit for bit launch_tsb_right_mul followed by launch_tsb_tn(W, W).
void launch_tsb_mul_gram(int n, int b, double *W, int64_t ldw, const double *Rinv, double *G,
                         const BlockScratch &bs, cudaStream_t st);
// Gram matrix G (b x b) of a block -> Rinv (b x b, upper triangular) with
// G = R^T R, by a Cholesky of the column-scaled G.  status[0] receives a
// bit mask of dependent columns: column j is dependent when its norm is
// <= abs_floor or its scaled pivot is <= rel_floor; such a column gets a
// unit pivot (it is replaced by the caller).  status[1] = 1 if any column
// is dependent, and then status[2] = 1 as well (status[2] is never cleared
// here: it records a dependency over several calls).  One warp.
void launch_block_chol(int b, const double *G, int ldg, double *Rinv, double abs_floor,
                       double rel_floor, int *status, cudaStream_t st);
// W[:, 0:b] = W[:, 0:b] Rinv  (in place; Rinv upper triangular b x b, ld b)
void launch_tsb_right_mul(int n, int b, double *W, int64_t ldw, const double *Rinv,
                          cudaStream_t st);
// W[:, 0:b] = X[:, 0:K] S  (S: K x b, leading dimension lds; K <= kBlockMaxM; W and X
// distinct)
void launch_tsb_right_mul_into(int n, int K, const double *X, int64_t ldx, const double *S,
                               int lds, double *W, int64_t ldw, int b, cudaStream_t st);

// FP64 refinement residual of a block solve:
//   R = B - (A + shift I) Y   (columns 0..b-1), and *flag <- 1 once every
//   column satisfies ||r_c|| <= tol * (anorm ||y_c|| + ||b_c||); while the
//   flag is 0, each evaluation adds one to *count (a correction follows).
// Does nothing when *flag is set.  part: >= 96 * ceil(n / 256) doubles;
// counter: one word, zero between launches.
void launch_block_refine_residual(int n, const int32_t *rowptr, const int32_t *col,
                                  const double *val, double shift, const double *B, int64_t ldb,
                                  const double *Y, int64_t ldy, double *R, int64_t ldr, int b,
                                  double tol, double anorm, int *flag, int *count, double *part,
                                  unsigned *counter, cudaStream_t st);
// Y[:, 0:b] += D[:, 0:b] unless *flag (flag may be null)
void launch_block_axpy_unless(int n, int b, double *Y, int64_t ldy, const double *D,
                              int64_t ldd, const int *flag, cudaStream_t st);
// dst[:, 0:b] = src[:, 0:b]
void launch_block_copy(int n, int b, const double *src, int64_t lds, double *dst, int64_t ldd,
                       cudaStream_t st);
// H[t + t * ldh] = theta[ord[t]] for t < l, the rest of the leading mm x mm
// part zero
void launch_block_set_diag(int ldh, int mm, int l, const double *theta, const int *ord,
                           double *H, cudaStream_t st);
// est[t]^2 = s_t^T G s_t with s_t = S[row0 : row0 + b, ord[t]] (the Ritz
// vector's coefficients on the last block) for t < nwant: the squared norm
// of the Ritz vector's residual under the block recurrence.
void launch_block_ritz_est(int nwant, int b, const double *S, int lds, int row0, const int *ord,
                           const double *G, int ldg, double *est2, cudaStream_t st);

}  // namespace spx
