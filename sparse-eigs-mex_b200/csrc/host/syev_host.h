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

}  // namespace spx
