// The projected eigenproblem of the Lanczos loops, on a host core.
//
// The reference solves its projected problem (order m = ncv, at most a few
// hundred) with LAPACK dsyev("V", "U") on the host (src/speigs_core.c:180,
// :236).  The same split is kept here: the m x m matrix is read back from the
// device, solved by Householder tridiagonalisation and the implicit
// symmetric QR iteration with Wilkinson shifts (Golub & Van Loan, Matrix
// Computations, 4th ed., algorithms 8.3.1 and 8.3.3), and the Ritz values,
// vectors and order are copied back.  At m = 33 to 128 this takes tens to a
// few hundred microseconds, where a one-block Jacobi on the device took
// 0.5 to 20 ms: the problem is a long chain of dependent rotations, which a
// single host core runs at full clock and an SM runs barrier by barrier.
#include "syev_host.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace spx {

namespace {

// A (n x n, column-major, full symmetric) -> tridiagonal (d, e) and the
// orthogonal Q with A = Q T Q^T.  Householder reflector k maps column k
// below the diagonal onto a multiple of the first unit vector.
void tridiagonalise(int n, std::vector<double> &A, std::vector<double> &d, std::vector<double> &e,
                    std::vector<double> &Q) {
    std::vector<double> v(n), p(n), beta(std::max(n - 2, 0), 0.0), V((size_t)n * n, 0.0);
    auto a = [&](int i, int j) -> double & { return A[(size_t)i + (size_t)j * n]; };
    for (int k = 0; k + 2 < n; k++) {
        const int L = n - k - 1;
        double sq = 0.0;
        for (int i = 0; i < L; i++) sq += a(k + 1 + i, k) * a(k + 1 + i, k);
        const double xn = std::sqrt(sq);
        if (xn == 0.0) continue;                   // column already reduced
        const double x0 = a(k + 1, k);
        const double alpha = x0 >= 0.0 ? -xn : xn;
        for (int i = 0; i < L; i++) v[i] = a(k + 1 + i, k);
        v[0] -= alpha;
        double vv = 0.0;
        for (int i = 0; i < L; i++) vv += v[i] * v[i];
        if (vv == 0.0) continue;
        const double b = 2.0 / vv;
        beta[k] = b;
        for (int i = 0; i < L; i++) V[(size_t)(k + 1 + i) + (size_t)k * n] = v[i];
        // p = b A22 v (A22 symmetric, full storage)
        for (int i = 0; i < L; i++) p[i] = 0.0;
        for (int j = 0; j < L; j++) {
            const double vj = b * v[j];
            const double *col = &A[(size_t)(k + 1) + (size_t)(k + 1 + j) * n];
            for (int i = 0; i < L; i++) p[i] += col[i] * vj;
        }
        double pv = 0.0;
        for (int i = 0; i < L; i++) pv += p[i] * v[i];
        const double K = 0.5 * b * pv;
        for (int i = 0; i < L; i++) p[i] -= K * v[i];      // w
        for (int j = 0; j < L; j++) {
            double *col = &A[(size_t)(k + 1) + (size_t)(k + 1 + j) * n];
            const double vj = v[j], wj = p[j];
            for (int i = 0; i < L; i++) col[i] -= v[i] * wj + p[i] * vj;
        }
        a(k + 1, k) = alpha;
        a(k, k + 1) = alpha;
        for (int i = 1; i < L; i++) a(k + 1 + i, k) = a(k, k + 1 + i) = 0.0;
    }
    d.assign(n, 0.0);
    e.assign(std::max(n - 1, 0), 0.0);
    for (int i = 0; i < n; i++) d[i] = a(i, i);
    for (int i = 0; i + 1 < n; i++) e[i] = a(i + 1, i);
    // Q = H_0 H_1 ... H_{n-3}, accumulated from the last reflector backward
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Q[(size_t)i + (size_t)i * n] = 1.0;
    std::vector<double> t(n);
    for (int k = n - 3; k >= 0; k--) {
        const double b = beta[k];
        if (b == 0.0) continue;
        const int L = n - k - 1;
        const double *vk = &V[(size_t)(k + 1) + (size_t)k * n];
        for (int j = 0; j < L; j++) {
            double *col = &Q[(size_t)(k + 1) + (size_t)(k + 1 + j) * n];
            double s = 0.0;
            for (int i = 0; i < L; i++) s += vk[i] * col[i];
            s *= b;
            for (int i = 0; i < L; i++) col[i] -= s * vk[i];
        }
    }
}

// Implicit symmetric QR on (d, e), rotations accumulated into the columns
// of Z (n x n).  Returns the number of QR steps, or -1 without convergence.
int tridiagonal_qr(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &Z) {
    const int max_steps = 30 * std::max(n, 1);
    int steps = 0;
    int hi = n - 1;
    while (hi > 0) {
        // deflate: negligible off-diagonals are set to zero
        for (int i = 0; i < hi; i++)
            if (std::fabs(e[i]) <= DBL_EPSILON * (std::fabs(d[i]) + std::fabs(d[i + 1]))) e[i] = 0.0;
        while (hi > 0 && e[hi - 1] == 0.0) hi--;
        if (hi == 0) break;
        int lo = hi - 1;
        while (lo > 0 && e[lo - 1] != 0.0) lo--;
        if (++steps > max_steps) return -1;
        // Wilkinson shift from the trailing 2 x 2 of the unreduced block
        const double dl = 0.5 * (d[hi - 1] - d[hi]);
        const double eh = e[hi - 1];
        const double den = dl + (dl >= 0.0 ? 1.0 : -1.0) * std::hypot(dl, eh);
        const double mu = den != 0.0 ? d[hi] - eh * eh / den : d[hi];
        double f = d[lo] - mu, h = e[lo], bulge = 0.0;
        for (int k = lo; k < hi; k++) {
            if (k > lo) {
                f = e[k - 1];
                h = bulge;
            }
            const double r = std::hypot(f, h);
            double c = 1.0, s = 0.0;
            if (r != 0.0) {
                c = f / r;
                s = h / r;
            }
            if (k > lo) e[k - 1] = r;
            const double p = d[k], q = d[k + 1], ek = e[k];
            d[k] = c * c * p + 2.0 * c * s * ek + s * s * q;
            d[k + 1] = s * s * p - 2.0 * c * s * ek + c * c * q;
            e[k] = c * s * (q - p) + (c * c - s * s) * ek;
            if (k + 1 < hi) {
                bulge = s * e[k + 1];
                e[k + 1] *= c;
            }
            double *zk = &Z[(size_t)k * n], *zk1 = &Z[(size_t)(k + 1) * n];
            for (int i = 0; i < n; i++) {
                const double a = zk[i], b = zk1[i];
                zk[i] = c * a + s * b;
                zk1[i] = c * b - s * a;
            }
        }
    }
    return steps;
}

}  // namespace

int syev_host(int m, const double *H, int ldh, double *theta, double *S, int *ord) {
    if (m <= 0) return 0;
    std::vector<double> A((size_t)m * m), d, e, Z;
    // the upper triangle, as dsyev("V", "U") reads it
    for (int j = 0; j < m; j++)
        for (int i = 0; i <= j; i++) {
            const double v = H[(size_t)i + (size_t)j * ldh];
            A[(size_t)i + (size_t)j * m] = v;
            A[(size_t)j + (size_t)i * m] = v;
        }
    tridiagonalise(m, A, d, e, Z);
    const int steps = tridiagonal_qr(m, d, e, Z);
    if (steps < 0) return -1;
    // ascending eigenvalues (stable), then the order by |theta| descending (stable)
    std::vector<int> pos(m);
    std::iota(pos.begin(), pos.end(), 0);
    std::stable_sort(pos.begin(), pos.end(), [&](int a, int b) { return d[a] < d[b]; });
    for (int i = 0; i < m; i++) {
        theta[i] = d[pos[i]];
        std::memcpy(S + (size_t)i * m, &Z[(size_t)pos[i] * m], sizeof(double) * m);
    }
    std::iota(ord, ord + m, 0);
    std::stable_sort(ord, ord + m,
                     [&](int a, int b) { return std::fabs(theta[a]) > std::fabs(theta[b]); });
    return steps;
}

}  // namespace spx

extern "C" int speigs_b200_syev_small_host(int m, const double *H, int ldh, double *theta,
                                           double *S, int *ord) {
    if (m <= 0 || ldh < m || !H || !theta || !S || !ord) return -1;
    return spx::syev_host(m, H, ldh, theta, S, ord) < 0 ? -1 : 0;
}
