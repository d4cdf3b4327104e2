// Complex Hermitian entry point through the real embedding (reference
// speigs_z, src/speigs_core.c:660-768).  For A = R + i S (R symmetric, S
// skew-symmetric) the real 2n x 2n matrix E = [[R, -S], [S, R]] is
// symmetric, and A (x + i y) = lambda (x + i y) exactly when E [x; y] =
// lambda [x; y]; every eigenvalue of A appears twice in E, through [x; y]
// and i (x + i y) = [-y; x].  The embedded problem runs through speigs() on
// the device (every route: diagonal, dense, components, banded, Krylov), and
// the complex eigenvectors are recovered on the device as well, the second
// copy of each eigenvalue dropped by complex Gram-Schmidt
// (spx::device_hermitian_recover).
#include "../engine.h"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

namespace {

// E in CSC with the numerically nonzero entries only: column j of E is
// [R(:, j); S(:, j)] and column n + j is [-S(:, j); R(:, j)].  Each column's
// length is counted first; then both halves of every column are written at
// their offsets in one pass over the input.
void embed(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Axr, const double *Axi,
           std::vector<int64_t> &Ep, std::vector<int64_t> &Ei, std::vector<double> &Ex) {
    Ep.assign(2 * n + 1, 0);
    std::vector<int64_t> nr(n), ns(n);
    for (int64_t j = 0; j < n; j++) {
        int64_t r = 0, s = 0;
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++) {
            r += Axr[q] != 0.0;
            s += Axi[q] != 0.0;
        }
        nr[j] = r;
        ns[j] = s;
        Ep[j + 1] = r + s;        // column j
        Ep[n + j + 1] = r + s;    // column n + j
    }
    for (int64_t c = 0; c < 2 * n; c++) Ep[c + 1] += Ep[c];
    Ei.assign(std::max<int64_t>(Ep[2 * n], 1), 0);
    Ex.assign(std::max<int64_t>(Ep[2 * n], 1), 0.0);
    for (int64_t j = 0; j < n; j++) {
        int64_t a = Ep[j], b = Ep[j] + nr[j];          // column j: R block, then S block
        int64_t c = Ep[n + j], d = Ep[n + j] + ns[j];  // column n + j: -S block, then R block
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++) {
            const int64_t i = Ai[q];
            if (Axr[q] != 0.0) {
                Ei[a] = i;     Ex[a++] = Axr[q];
                Ei[d] = n + i; Ex[d++] = Axr[q];
            }
            if (Axi[q] != 0.0) {
                Ei[b] = n + i; Ex[b++] = Axi[q];
                Ei[c] = i;     Ex[c++] = -Axi[q];
            }
        }
    }
}

}  // namespace

extern "C" int speigs_z(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                        const double *Axr, const double *Axi, speigs_int k, speigs_which which,
                        const speigs_opts *opts, double *lambda, double *Vr, double *Vi,
                        double *resid, speigs_info *info) {
    if (!Axi) return speigs(n, Ap, Ai, Axr, k, which, opts, lambda, Vr, resid, info);
    speigs_info li;
    if (!info) info = &li;
    if (n <= 0 || k <= 0 || k > n || !Ap || !Ai || !Axr || !lambda) return SPEIGS_ERR_ARG;
    std::vector<int64_t> Ep, Ei;
    std::vector<double> Ex;
    embed(n, Ap, Ai, Axr, Axi, Ep, Ei, Ex);
    // each wanted eigenvalue appears twice in the embedding: ask for 2k + 2
    const int64_t n2 = 2 * n, kk = std::min<int64_t>(2 * k + 2, n2);
    std::vector<double> lam2(kk), res2(kk), V2((size_t)n2 * kk);
    int rc = speigs(n2, Ep.data(), Ei.data(), Ex.data(), kk, which, opts, lam2.data(), V2.data(),
                    res2.data(), info);
    if (rc) return rc;
    int64_t nacc = 0;
    rc = spx::device_hermitian_recover(n, kk, k, V2.data(), lam2.data(), res2.data(), lambda, Vr,
                                       Vi, resid, &nacc);
    if (rc) return rc;
    info->nconv = nacc;
    if (nacc < k) info->flag = 1;
    return SPEIGS_OK;
}
