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
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace spx {

namespace {

// A (n x n, column-major, full symmetric) -> tridiagonal (d, e) with
// A = Q T Q^T, Q = H_0 H_1 ... H_{n-3}.  Householder reflector H_k =
// I - beta[k] v_k v_k^T maps column k below the diagonal onto a multiple of
// the first unit vector; v_k is kept in column k of V (rows k+1 .. n-1).
void reduce(int n, std::vector<double> &A, std::vector<double> &d, std::vector<double> &e,
            std::vector<double> &V, std::vector<double> &beta) {
    std::vector<double> v(n), p(n);
    beta.assign(std::max(n - 2, 0), 0.0);
    V.assign((size_t)n * n, 0.0);
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
}

// Q = H_0 H_1 ... H_{n-3}, accumulated from the last reflector backward
void form_q(int n, const std::vector<double> &V, const std::vector<double> &beta,
            std::vector<double> &Q) {
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Q[(size_t)i + (size_t)i * n] = 1.0;
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

// The reduction of `reduce` reading and updating only the lower triangle of
// A: p = beta A22 v as one symmetric pass (each stored entry used twice),
// then the rank-2 update of the lower triangle -- 2 L^2 multiply-adds a
// step instead of 3 L^2.  Same reflectors up to rounding.
void reduce_lower(int n, std::vector<double> &A, std::vector<double> &d, std::vector<double> &e,
                  std::vector<double> &V, std::vector<double> &beta) {
    std::vector<double> v(n), p(n);
    beta.assign(std::max(n - 2, 0), 0.0);
    V.assign((size_t)n * n, 0.0);
    auto a = [&](int i, int j) -> double & { return A[(size_t)i + (size_t)j * n]; };
    for (int k = 0; k + 2 < n; k++) {
        const int L = n - k - 1;
        const double *x = &A[(size_t)(k + 1) + (size_t)k * n];
        double sq = 0.0;
        for (int i = 0; i < L; i++) sq += x[i] * x[i];
        const double xn = std::sqrt(sq);
        if (xn == 0.0) continue;
        const double alpha = x[0] >= 0.0 ? -xn : xn;
        for (int i = 0; i < L; i++) v[i] = x[i];
        v[0] -= alpha;
        double vv = 0.0;
        for (int i = 0; i < L; i++) vv += v[i] * v[i];
        if (vv == 0.0) continue;
        const double b = 2.0 / vv;
        beta[k] = b;
        std::memcpy(&V[(size_t)(k + 1) + (size_t)k * n], v.data(), sizeof(double) * L);
        for (int i = 0; i < L; i++) p[i] = 0.0;
        for (int j = 0; j < L; j++) {
            const double *col = &A[(size_t)(k + 1) + (size_t)(k + 1 + j) * n];
            const double vj = v[j];
            double acc = col[j] * vj;
            for (int i = j + 1; i < L; i++) {
                p[i] += col[i] * vj;
                acc += col[i] * v[i];
            }
            p[j] += acc;
        }
        double pv = 0.0;
        for (int i = 0; i < L; i++) {
            p[i] *= b;
            pv += p[i] * v[i];
        }
        const double K = 0.5 * b * pv;
        for (int i = 0; i < L; i++) p[i] -= K * v[i];      // w
        for (int j = 0; j < L; j++) {
            double *col = &A[(size_t)(k + 1) + (size_t)(k + 1 + j) * n];
            const double vj = v[j], wj = p[j];
            for (int i = j; i < L; i++) col[i] -= v[i] * wj + p[i] * vj;
        }
        a(k + 1, k) = alpha;
    }
    d.assign(n, 0.0);
    e.assign(std::max(n - 1, 0), 0.0);
    for (int i = 0; i < n; i++) d[i] = a(i, i);
    for (int i = 0; i + 1 < n; i++) e[i] = a(i + 1, i);
}

// sqrt(f^2 + h^2): the plain formula inside a range where it cannot
// overflow or lose the smaller term to underflow, std::hypot outside it
inline double rot_norm(double f, double h) {
    const double mx = std::max(std::fabs(f), std::fabs(h));
    if (mx > 1e-150 && mx < 1e150) return std::sqrt(f * f + h * h);
    return std::hypot(f, h);
}

// Implicit symmetric QR on (d, e), rotations accumulated into the columns
// of Z (n x n) when Z is given.  Without Z (eigenvalues only) the rotation
// lengths use rot_norm instead of std::hypot, which rounds differently in
// the last bit.  Returns the number of QR steps, or -1 without convergence.
int tridiagonal_qr(int n, std::vector<double> &d, std::vector<double> &e, double *Z) {
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
            const double r = Z ? std::hypot(f, h) : rot_norm(f, h);
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
            if (!Z) continue;
            double *zk = Z + (size_t)k * n, *zk1 = Z + (size_t)(k + 1) * n;
            for (int i = 0; i < n; i++) {
                const double a = zk[i], b = zk1[i];
                zk[i] = c * a + s * b;
                zk1[i] = c * b - s * a;
            }
        }
    }
    return steps;
}

// Z := Q Z = H_0 H_1 ... H_{n-3} Z for the nc columns of Z (leading
// dimension n), the reflectors applied from the last
void apply_q(int n, const std::vector<double> &V, const std::vector<double> &beta, double *Z,
             int nc) {
    for (int k = n - 3; k >= 0; k--) {
        const double b = beta[k];
        if (b == 0.0) continue;
        const int L = n - k - 1;
        const double *vk = &V[(size_t)(k + 1) + (size_t)k * n];
        for (int c = 0; c < nc; c++) {
            double *z = Z + (size_t)c * n + k + 1;
            double s = 0.0;
            for (int i = 0; i < L; i++) s += vk[i] * z[i];
            s *= b;
            for (int i = 0; i < L; i++) z[i] -= s * vk[i];
        }
    }
}

// Gaussian elimination with partial pivoting of the tridiagonal T - sigma I
// (diagonal d - sigma, both off-diagonals e): row i of U holds u0[i] on the
// diagonal and u1[i], u2[i] on the next two columns; step i eliminated
// below the pivot with multiplier l[i] after swapping rows i and i+1 when
// swp[i].  A pivot that vanishes is replaced by `tiny`.
struct TriLU {
    std::vector<double> u0, u1, u2, l;
    std::vector<char> swp;
    void factor(int n, const std::vector<double> &d, const std::vector<double> &e, double sigma,
                double tiny) {
        u0.assign(n, 0.0); u1.assign(n, 0.0); u2.assign(n, 0.0); l.assign(n, 0.0);
        swp.assign(n, 0);
        // pending row i: x0 (column i), x1 (i+1), x2 (i+2)
        double x0 = d[0] - sigma, x1 = n > 1 ? e[0] : 0.0, x2 = 0.0;
        for (int i = 0; i + 1 < n; i++) {
            const double sub = e[i], dn = d[i + 1] - sigma, sn = i + 2 < n ? e[i + 1] : 0.0;
            if (std::fabs(x0) >= std::fabs(sub)) {
                if (x0 == 0.0) x0 = tiny;
                const double m = sub / x0;
                u0[i] = x0; u1[i] = x1; u2[i] = x2; l[i] = m;
                x0 = dn - m * x1;
                x1 = sn - m * x2;
            } else {
                const double m = x0 / sub;
                u0[i] = sub; u1[i] = dn; u2[i] = sn; l[i] = m; swp[i] = 1;
                x0 = x1 - m * dn;
                x1 = x2 - m * sn;
            }
            x2 = 0.0;
        }
        u0[n - 1] = x0 == 0.0 ? tiny : x0;
    }
    // y := (T - sigma I)^{-1} y
    void solve(int n, double *y) const {
        for (int i = 0; i + 1 < n; i++) {
            if (swp[i]) std::swap(y[i], y[i + 1]);
            y[i + 1] -= l[i] * y[i];
        }
        y[n - 1] /= u0[n - 1];
        if (n >= 2) y[n - 2] = (y[n - 2] - u1[n - 2] * y[n - 1]) / u0[n - 2];
        for (int i = n - 3; i >= 0; i--) y[i] = (y[i] - u1[i] * y[i + 1] - u2[i] * y[i + 2]) / u0[i];
    }
};

}  // namespace

int syev_host_select(int m, const double *H, int ldh, int nvec, double *theta, double *S,
                     int *ord) {
    if (m <= 0) return 0;
    if (nvec >= m) return syev_host(m, H, ldh, theta, S, ord);
    std::vector<double> A((size_t)m * m), d, e, V, beta;
    for (int j = 0; j < m; j++)
        for (int i = 0; i <= j; i++) {
            const double v = H[(size_t)i + (size_t)j * ldh];
            A[(size_t)i + (size_t)j * m] = v;
            A[(size_t)j + (size_t)i * m] = v;
        }
    reduce_lower(m, A, d, e, V, beta);
    const std::vector<double> d0 = d, e0 = e;      // T, for the inverse iteration
    const int steps = tridiagonal_qr(m, d, e, nullptr);
    if (steps < 0) return -1;
    std::vector<int> pos(m);
    std::iota(pos.begin(), pos.end(), 0);
    std::stable_sort(pos.begin(), pos.end(), [&](int a, int b) { return d[a] < d[b]; });
    for (int i = 0; i < m; i++) theta[i] = d[pos[i]];
    std::iota(ord, ord + m, 0);
    std::stable_sort(ord, ord + m,
                     [&](int a, int b) { return std::fabs(theta[a]) > std::fabs(theta[b]); });
    std::memset(S, 0, sizeof(double) * (size_t)m * m);
    if (nvec <= 0) return steps;
    // the wanted eigenvalues in ascending order; a cluster is a run whose
    // neighbours lie within 1e-3 ||T||_inf, and each vector is kept
    // orthogonal to those computed before it in its cluster
    std::vector<int> want(ord, ord + nvec);
    std::sort(want.begin(), want.end());
    double tnorm = 0.0;
    for (int i = 0; i < m; i++)
        tnorm = std::max(tnorm, std::fabs(d0[i]) + (i > 0 ? std::fabs(e0[i - 1]) : 0.0) +
                                    (i + 1 < m ? std::fabs(e0[i]) : 0.0));
    if (tnorm == 0.0) tnorm = 1.0;
    const double tiny = DBL_EPSILON * tnorm, ortol = 1e-3 * tnorm;
    TriLU lu;
    std::vector<double> z(m), Zw((size_t)m * want.size());
    std::vector<std::vector<double>> clus;          // eigenvectors of T in the current cluster
    uint64_t rs = 0x9E3779B97F4A7C15ULL;
    for (size_t w = 0; w < want.size(); w++) {
        const int j = want[w];
        if (w == 0 || theta[j] - theta[want[w - 1]] > ortol) clus.clear();
        lu.factor(m, d0, e0, theta[j], tiny);
        for (int i = 0; i < m; i++) {                // start: uniform in [-1, 1] (xorshift64*)
            rs ^= rs >> 12; rs ^= rs << 25; rs ^= rs >> 27;
            z[i] = 2.0 * (double)((rs * 0x2545F4914F6CDD1DULL) >> 11) / 9007199254740992.0 - 1.0;
        }
        for (int it = 0; it < 3; it++) {
            double mx = 0.0;
            for (int i = 0; i < m; i++) mx = std::max(mx, std::fabs(z[i]));
            for (int i = 0; i < m; i++) z[i] /= mx;
            lu.solve(m, z.data());
            for (const auto &q : clus) {
                double dot = 0.0;
                for (int i = 0; i < m; i++) dot += q[i] * z[i];
                for (int i = 0; i < m; i++) z[i] -= dot * q[i];
            }
        }
        double nrm = 0.0;
        for (int i = 0; i < m; i++) nrm += z[i] * z[i];
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return -1;
        for (int i = 0; i < m; i++) z[i] /= nrm;
        clus.push_back(z);
        std::memcpy(Zw.data() + w * m, z.data(), sizeof(double) * m);
    }
    apply_q(m, V, beta, Zw.data(), (int)want.size());
    for (size_t w = 0; w < want.size(); w++)
        std::memcpy(S + (size_t)want[w] * m, Zw.data() + w * m, sizeof(double) * m);
    return steps;
}

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
    std::vector<double> V, beta;
    reduce(m, A, d, e, V, beta);
    form_q(m, V, beta, Z);
    const int steps = tridiagonal_qr(m, d, e, Z.data());
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

extern "C" int speigs_b200_syev_select_host(int m, const double *H, int ldh, int nvec,
                                            double *theta, double *S, int *ord) {
    if (m <= 0 || ldh < m || nvec < 0 || !H || !theta || !S || !ord) return -1;
    return spx::syev_host_select(m, H, ldh, nvec, theta, S, ord) < 0 ? -1 : 0;
}
