// Host solver of the Lanczos loops' projected eigenproblem (syev_host.cpp).
#pragma once

namespace spx {

// Eigen-decomposition of the symmetric m x m matrix whose upper triangle is
// H (column-major, leading dimension ldh): theta ascending, S (m x m, ld m)
// the matching eigenvectors, ord[t] the index into theta of the t-th
// largest |theta| (ties keep ascending order) -- the contract of the
// device Jacobi (launch_syev_small).  Returns the QR steps taken, or -1 when
// the iteration did not converge in 30 m steps.
int syev_host(int m, const double *H, int ldh, double *theta, double *S, int *ord);

// The same theta and ord, with eigenvectors only for the nvec leading
// entries of ord (the other columns of S are zero): Householder reduction
// of the lower triangle, implicit QR on the eigenvalues alone (theta agrees
// with syev_host's to rounding), inverse iteration on the tridiagonal
// for the wanted eigenvalues with Gram-Schmidt against the earlier vectors
// of a cluster (neighbours within 1e-3 ||T||_inf), and the reflectors
// applied to the results -- the method of LAPACK's dsyevx (dstebz/dstein/
// dormtr), at O(m^2) per vector instead of the O(m^3) accumulation.
// nvec >= m is syev_host.  Returns the QR steps, or -1.
int syev_host_select(int m, const double *H, int ldh, int nvec, double *theta, double *S,
                     int *ord);

}  // namespace spx
