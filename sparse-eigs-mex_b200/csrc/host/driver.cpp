// C API of libspeigs: argument checks, structure analysis and routing, then
// the device engine.  Mirrors the reference driver speigs()
// (src/speigs_core.c:783-1024) route for route:
//   symmetry check (:795) -> diagonal (:801) -> dense gate (:806) ->
//   connected components (:814-827) -> ||A||_1 (:840) -> 'lm' direct or
//   'sm' shift-invert with the capped shift escalation (:938-970) ->
//   Lanczos (:990) -> output sorted by |lambda| (:994-1012).
// Host work here is setup only (pattern checks, union-find, ordering); every
// numerical step of every route runs on the GPU.
#include "../engine.h"
#include "../../../include/speigs_b200.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <vector>

using spx::HostCSR;

namespace {

double wall() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

// 1: symmetric with both triangles, 2: upper only, 3: lower only, 0: not
// symmetric (reference check_symmetry, src/speigs_core.c:363-401; transposed
// entries must agree to 1e-12 relative).
int check_symmetry(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax) {
    bool up = false, lo = false;
    for (int64_t c = 0; c < n && !(up && lo); c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            if (Ai[q] < c) up = true;
            else if (Ai[q] > c) lo = true;
        }
    if (!lo && up) return 2;
    if (!up && lo) return 3;
    if (!up && !lo) return 1;
    const int64_t nnz = Ap[n];
    std::vector<int64_t> Tp(n + 1, 0), Ti(nnz ? nnz : 1), wk(n, 0);
    std::vector<double> Tx(nnz ? nnz : 1);
    for (int64_t q = 0; q < nnz; q++) wk[Ai[q]]++;
    for (int64_t i = 0; i < n; i++) { Tp[i + 1] = Tp[i] + wk[i]; wk[i] = Tp[i]; }
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            int64_t d = wk[Ai[q]]++;
            Ti[d] = c;
            Tx[d] = Ax[q];
        }
    for (int64_t i = 0; i <= n; i++) if (Tp[i] != Ap[i]) return 0;
    for (int64_t q = 0; q < nnz; q++) {
        if (Ti[q] != Ai[q]) return 0;
        const double a = Ax[q], b = Tx[q];
        const double m = std::max(fabs(a), fabs(b));
        if (fabs(a - b) > 1e-12 * (m > 0 ? m : 1.0)) return 0;
    }
    return 1;
}

bool is_diagonal(int64_t n, const int64_t *Ap, const int64_t *Ai) {
    for (int64_t c = 0; c < n; c++)
        for (int64_t p = Ap[c]; p < Ap[c + 1]; p++)
            if (Ai[p] != c) return false;
    return true;
}

int64_t uf_find(std::vector<int64_t> &p, int64_t x) {
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}

// Components over the numerically nonzero entries (reference
// find_components, src/speigs_core.c:445-466): labels in order of first
// appearance.
int64_t find_components(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                        std::vector<int64_t> &comp) {
    std::vector<int64_t> p(n);
    for (int64_t i = 0; i < n; i++) p[i] = i;
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++)
            if (Ax[q] != 0.0) {
                int64_t a = uf_find(p, Ai[q]), b = uf_find(p, c);
                if (a != b) p[a] = b;
            }
    std::vector<int64_t> lab(n, -1);
    comp.assign(n, 0);
    int64_t nc = 0;
    for (int64_t i = 0; i < n; i++) {
        int64_t r = uf_find(p, i);
        if (lab[r] < 0) lab[r] = nc++;
        comp[i] = lab[r];
    }
    return nc;
}

// ||A||_1 of the symmetric matrix of the upper triangle (cholmod_l_norm_sparse
// with stype = 1, as the reference calls it at src/speigs_core.c:840).
double norm1_upper(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax) {
    std::vector<double> s(n, 0.0);
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            const int64_t r = Ai[q];
            if (r > c) continue;
            s[c] += fabs(Ax[q]);
            if (r != c) s[r] += fabs(Ax[q]);
        }
    double m = 0;
    for (double v : s) m = std::max(m, v);
    return m;
}

struct Cand { double key; int64_t idx; };

int speigs_impl(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax, int64_t k,
                speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                double *lambda, double *V, double *resid, speigs_info *info,
                speigs_ext_info *einfo);

// Solve every component separately and merge by |lambda| (reference
// blocks_path, src/speigs_core.c:532-632).
int blocks_path(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax, int64_t k,
                speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                const std::vector<int64_t> &comp, int64_t ncomp, double *lambda, double *V,
                double *resid, speigs_info *info, speigs_ext_info *einfo) {
    std::vector<int64_t> sz(ncomp, 0), off(ncomp + 1, 0), gidx(n), loc(n), fill(ncomp, 0);
    for (int64_t i = 0; i < n; i++) sz[comp[i]]++;
    for (int64_t c = 0; c < ncomp; c++) off[c + 1] = off[c] + sz[c];
    for (int64_t i = 0; i < n; i++) {
        const int64_t c = comp[i], slot = off[c] + fill[c]++;
        gidx[slot] = i;
        loc[i] = slot - off[c];
    }
    std::vector<double> clam, cres;
    std::vector<int64_t> ccomp, cslot;
    std::vector<std::vector<double>> cvec(ncomp);
    std::vector<int64_t> sAp(n + 1), sAi(Ap[n] ? Ap[n] : 1);
    std::vector<double> sAx(Ap[n] ? Ap[n] : 1);
    for (int64_t ci = 0; ci < ncomp; ci++) {
        const int64_t nc = sz[ci];
        int64_t knt = 0;
        for (int64_t j = 0; j < nc; j++) {
            const int64_t gc = gidx[off[ci] + j];
            sAp[j] = knt;
            for (int64_t q = Ap[gc]; q < Ap[gc + 1]; q++) {
                const int64_t r = Ai[q];
                if (comp[r] == ci) { sAi[knt] = loc[r]; sAx[knt] = Ax[q]; knt++; }
            }
        }
        sAp[nc] = knt;
        const int64_t kc = std::min(k, nc);
        std::vector<double> lv(kc), rv(kc);
        if (V) cvec[ci].assign((size_t)nc * kc, 0.0);
        speigs_info si;
        speigs_ext_info se;
        int r2 = speigs_impl(nc, sAp.data(), sAi.data(), sAx.data(), kc, which, opts, ext,
                             lv.data(), V ? cvec[ci].data() : nullptr, rv.data(), &si, &se);
        if (r2) return r2;
        if (einfo) {
            einfo->refine_steps += se.refine_steps;
            einfo->factor_solves += se.factor_solves;
            if (se.precision) einfo->precision = se.precision;
        }
        info->nops += si.nops;
        if (si.flag) info->flag = 1;
        for (int64_t t = 0; t < kc; t++) {
            clam.push_back(lv[t]);
            cres.push_back(rv[t]);
            ccomp.push_back(ci);
            cslot.push_back(t);
        }
    }
    const int64_t ncand = (int64_t)clam.size();
    std::vector<Cand> ord(ncand);
    for (int64_t i = 0; i < ncand; i++) ord[i] = {fabs(clam[i]), i};
    std::stable_sort(ord.begin(), ord.end(), [&](const Cand &a, const Cand &b) {
        return which == SPEIGS_SM ? a.key < b.key : a.key > b.key;
    });
    for (int64_t t = 0; t < k && t < ncand; t++) {
        const int64_t i = ord[t].idx, ci = ccomp[i], sl = cslot[i], nc = sz[ci];
        lambda[t] = clam[i];
        if (resid) resid[t] = cres[i];
        if (V) {
            memset(V + (size_t)t * n, 0, (size_t)n * sizeof(double));
            const double *src = cvec[ci].data() + (size_t)sl * nc;
            for (int64_t j = 0; j < nc; j++) V[(size_t)t * n + gidx[off[ci] + j]] = src[j];
        }
    }
    info->nconv = std::min(k, ncand);
    info->ncomp = ncomp;
    info->path = SPEIGS_PATH_BLOCKS;
    return SPEIGS_OK;
}

}  // namespace

namespace spx {
int host_check_symmetry(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax) {
    return check_symmetry(n, Ap, Ai, Ax);
}
double host_norm1_upper(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax) {
    return norm1_upper(n, Ap, Ai, Ax);
}
}  // namespace spx

extern "C" {

void speigs_default_opts(speigs_opts *o) {
    memset(o, 0, sizeof *o);
    o->dense_max = -1;
    o->detect = 1;
    o->check_sym = 1;
}

const char *speigs_errmsg(int c) {
    switch (c) {
        case SPEIGS_OK: return "ok";
        case SPEIGS_ERR_ARG: return "invalid argument";
        case SPEIGS_ERR_MEM: return "out of memory";
        case SPEIGS_ERR_FACTOR: return "factorization failed";
        case SPEIGS_ERR_LAPACK: return "LAPACK failed";
        case SPEIGS_ERR_NOTSYM:
            return "matrix is not symmetric "
                   "(this solver is for symmetric/Hermitian matrices only)";
        default: return "internal error";
    }
}

int speigs(speigs_int n, const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
           speigs_int k, speigs_which which, const speigs_opts *opts, double *lambda, double *V,
           double *resid, speigs_info *info) {
    return speigs_impl(n, Ap, Ai, Ax, k, which, opts, nullptr, lambda, V, resid, info, nullptr);
}

int speigs_ex(speigs_int n, const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
              speigs_int k, speigs_which which, const speigs_opts *opts,
              const speigs_ext_opts *ext, double *lambda, double *V, double *resid,
              speigs_info *info, speigs_ext_info *einfo) {
    return speigs_impl(n, Ap, Ai, Ax, k, which, opts, ext, lambda, V, resid, info, einfo);
}

}  // extern "C"

namespace {

int speigs_impl(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax, int64_t k,
                speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                double *lambda, double *V, double *resid, speigs_info *info,
                speigs_ext_info *einfo) {
    speigs_ext_info le;
    if (!einfo) einfo = &le;
    memset(einfo, 0, sizeof *einfo);
    speigs_opts defo;
    if (!opts) { speigs_default_opts(&defo); opts = &defo; }
    speigs_info li;
    if (!info) info = &li;
    memset(info, 0, sizeof *info);
    if (n <= 0 || !Ap || !Ai || !Ax || !lambda) return SPEIGS_ERR_ARG;
    if (k <= 0 || k > n) return SPEIGS_ERR_ARG;
    if (opts->check_sym != 0 && check_symmetry(n, Ap, Ai, Ax) == 0) return SPEIGS_ERR_NOTSYM;

    const double t0 = wall();
    const int dmax = opts->dense_max < 0 ? 800 : opts->dense_max;
    if (opts->detect && is_diagonal(n, Ap, Ai)) {
        std::vector<double> d(n, 0.0);
        for (int64_t c = 0; c < n; c++)
            for (int64_t p = Ap[c]; p < Ap[c + 1]; p++) if (Ai[p] == c) d[c] = Ax[p];
        return spx::device_diag_path(n, d.data(), k, which, lambda, V, resid, info);
    }
    if (dmax > 0 && (n <= dmax || 4 * k > n)) {
        HostCSR A;
        int rc = spx::build_full_csr(n, Ap, Ai, Ax, &A);
        if (rc) return rc;
        rc = spx::device_dense_path(A, k, which, lambda, V, resid, info);
        spx::free_csr(&A);
        info->t_iter = wall() - t0;
        return rc;
    }
    if (opts->detect) {
        std::vector<int64_t> comp;
        const int64_t ncomp = find_components(n, Ap, Ai, Ax, comp);
        if (ncomp > 1) {
            int rc = blocks_path(n, Ap, Ai, Ax, k, which, opts, ext, comp, ncomp, lambda, V, resid,
                                 info, einfo);
            info->t_iter = wall() - t0;
            return rc;
        }
    }
    double anorm = norm1_upper(n, Ap, Ai, Ax);
    if (anorm <= 0) anorm = 1.0;
    info->anorm = anorm;
    HostCSR A;
    int rc = spx::build_full_csr(n, Ap, Ai, Ax, &A);
    if (rc) return rc;
    // factor + Lanczos on the device; results come back sorted by |lambda|
    return spx::device_krylov(A, k, which, *opts, anorm, lambda, V, resid, info, nullptr, ext,
                              einfo);
}

}  // namespace
