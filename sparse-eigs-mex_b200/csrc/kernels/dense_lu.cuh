// The indefinite route's operator: A^{-1} for a symmetric matrix that stays
// indefinite after the capped shift escalation (the reference factors A at
// sigma = 0 with UMFPACK, src/speigs_core.c:972-984, and applies the LU
// solve as its operator, :111-115).  Here the inverse is formed on the
// device by Gauss-Jordan elimination with partial (row) pivoting, and each
// operator application is one dense matrix-vector product.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spx {

// Largest order the route accepts (the dense inverse holds n^2 doubles).
constexpr int kLuDenseMax = 8192;

// M (n x n, column-major, ld n, device) = A^{-1} for the full symmetric CSR
// A.  Scratch (device): rowbuf[n], colbuf[n], ipiv[n] ints, flags[2] ints.
// A pivot that is exactly zero is replaced by eps * anorm and flags[0] is
// set (the matrix is singular to working precision); the other pivots are
// the largest entries of their columns.
void launch_dense_inverse(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                          double anorm, double *M, double *rowbuf, double *colbuf, int *ipiv,
                          int *flags, cudaStream_t st);

// y = M^T x for the dense inverse (a symmetric matrix, so either product is
// the operator; the transposed one reads M's columns contiguously).
void launch_dense_apply(int n, const double *M, const double *x, double *y, cudaStream_t st);

}  // namespace spx
