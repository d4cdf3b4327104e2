// Complex Hermitian entry point through the real 2n x 2n embedding
// [[R, -S], [S, R]] (reference speigs_z, src/speigs_core.c:660-768).  The
// embedded real problem runs through speigs() on the device; this file builds
// the embedding and recovers the complex eigenvectors, dropping the i-multiple
// duplicates by complex Gram-Schmidt (the reference's :708-757).
#include "../../../include/speigs.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

extern "C" int speigs_z(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                        const double *Axr, const double *Axi, speigs_int k, speigs_which which,
                        const speigs_opts *opts, double *lambda, double *Vr, double *Vi,
                        double *resid, speigs_info *info) {
    if (!Axi) return speigs(n, Ap, Ai, Axr, k, which, opts, lambda, Vr, resid, info);
    speigs_info li;
    if (!info) info = &li;
    if (n <= 0 || k <= 0 || k > n || !Ap || !Ai || !Axr || !lambda) return SPEIGS_ERR_ARG;
    const int64_t n2 = 2 * n, nnz = Ap[n];
    int64_t nzR = 0, nzS = 0;
    for (int64_t q = 0; q < nnz; q++) { nzR += (Axr[q] != 0.0); nzS += (Axi[q] != 0.0); }
    const int64_t nz2 = 2 * (nzR + nzS);
    std::vector<int64_t> Bp(n2 + 1), Bi(nz2 ? nz2 : 1);
    std::vector<double> Bx(nz2 ? nz2 : 1);
    int64_t t = 0;
    for (int64_t j = 0; j < n; j++) {            // column j: [R; S]
        Bp[j] = t;
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++)
            if (Axr[q] != 0.0) { Bi[t] = Ai[q]; Bx[t] = Axr[q]; t++; }
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++)
            if (Axi[q] != 0.0) { Bi[t] = n + Ai[q]; Bx[t] = Axi[q]; t++; }
    }
    for (int64_t j = 0; j < n; j++) {            // column n+j: [-S; R]
        Bp[n + j] = t;
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++)
            if (Axi[q] != 0.0) { Bi[t] = Ai[q]; Bx[t] = -Axi[q]; t++; }
        for (int64_t q = Ap[j]; q < Ap[j + 1]; q++)
            if (Axr[q] != 0.0) { Bi[t] = n + Ai[q]; Bx[t] = Axr[q]; t++; }
    }
    Bp[n2] = t;
    // every eigenvalue of A appears twice in the embedding
    const int64_t kk = std::min<int64_t>(2 * k + 2, n2);
    std::vector<double> lam2(kk), res2(kk), V2((size_t)n2 * kk);
    int rc = speigs(n2, Bp.data(), Bi.data(), Bx.data(), kk, which, opts, lam2.data(), V2.data(),
                    res2.data(), info);
    if (rc) return rc;
    std::vector<double> ar((size_t)n * k, 0.0), ai((size_t)n * k, 0.0), wr(n), wi(n);
    int64_t nacc = 0;
    for (int64_t c = 0; c < kk && nacc < k; c++) {
        const double *a = V2.data() + (size_t)c * n2, *b = a + n;
        double nr = 0.0;
        for (int64_t i = 0; i < n; i++) nr += a[i] * a[i] + b[i] * b[i];
        if (nr <= 0.0) continue;
        nr = 1.0 / sqrt(nr);
        for (int64_t i = 0; i < n; i++) { wr[i] = a[i] * nr; wi[i] = b[i] * nr; }
        for (int pass = 0; pass < 2; pass++)
            for (int64_t u = 0; u < nacc; u++) {
                const double *ur = ar.data() + (size_t)u * n, *ui = ai.data() + (size_t)u * n;
                double re = 0.0, im = 0.0;   // <u, w> = sum conj(u) w
                for (int64_t i = 0; i < n; i++) {
                    re += ur[i] * wr[i] + ui[i] * wi[i];
                    im += ur[i] * wi[i] - ui[i] * wr[i];
                }
                for (int64_t i = 0; i < n; i++) {
                    const double xr = ur[i], xi = ui[i];
                    wr[i] -= re * xr - im * xi;
                    wi[i] -= re * xi + im * xr;
                }
            }
        double wn = 0.0;
        for (int64_t i = 0; i < n; i++) wn += wr[i] * wr[i] + wi[i] * wi[i];
        wn = sqrt(wn);
        if (wn <= 0.1) continue;   // an i-multiple of an accepted vector
        const double inv = 1.0 / wn;
        for (int64_t i = 0; i < n; i++) {
            ar[(size_t)nacc * n + i] = wr[i] * inv;
            ai[(size_t)nacc * n + i] = wi[i] * inv;
        }
        lambda[nacc] = lam2[c];
        if (resid) resid[nacc] = res2[c];
        nacc++;
    }
    if (Vr) memcpy(Vr, ar.data(), (size_t)n * k * sizeof(double));
    if (Vi) memcpy(Vi, ai.data(), (size_t)n * k * sizeof(double));
    info->nconv = nacc;
    if (nacc < k) info->flag = 1;
    return SPEIGS_OK;
}
