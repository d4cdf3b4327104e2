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
#include "parallel.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <thread>
#include <utility>
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

// check_symmetry for large inputs: the same verdict, from parallel passes.
// When every column's row indices are strictly increasing, "the transpose
// equals A entry for entry" is "every (r, c) has its mirror (c, r), with a
// value within 1e-12 relative", which each column tests on its own by binary
// search; otherwise the transposition above decides.  *full_sorted is set
// when the verdict is 1 with both triangles stored and sorted columns.
int check_symmetry_par(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                       bool *full_sorted) {
    *full_sorted = false;
    std::atomic<int> up{0}, lo{0}, unsorted{0};
    spx::parallel_ranges(n, 8192, [&](int64_t c0, int64_t c1) {
        bool u = false, l = false, uns = false;
        for (int64_t c = c0; c < c1; c++)
            for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
                if (Ai[q] < c) u = true;
                else if (Ai[q] > c) l = true;
                if (q > Ap[c] && Ai[q] <= Ai[q - 1]) uns = true;
            }
        if (u) up = 1;
        if (l) lo = 1;
        if (uns) unsorted = 1;
    });
    if (!lo && up) return 2;
    if (!up && lo) return 3;
    if (!up && !lo) return 1;
    if (unsorted) return check_symmetry(n, Ap, Ai, Ax);
    std::atomic<int> bad{0};
    spx::parallel_ranges(n, 8192, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1 && !bad.load(std::memory_order_relaxed); c++)
            for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
                const int64_t r = Ai[q];
                if (r == c) continue;
                if (r < 0 || r >= n) { bad = 1; break; }
                const int64_t *b = Ai + Ap[r], *e = Ai + Ap[r + 1];
                const int64_t *f = std::lower_bound(b, e, c);
                if (f == e || *f != c) { bad = 1; break; }
                const double a = Ax[q], t = Ax[f - Ai];
                const double m = std::max(fabs(a), fabs(t));
                if (fabs(a - t) > 1e-12 * (m > 0 ? m : 1.0)) { bad = 1; break; }
            }
    });
    if (bad) return 0;
    *full_sorted = true;
    return 1;
}

// find_components for large inputs: the same labels (components over the
// numerically nonzero entries, numbered in order of first appearance), with
// the unions done in parallel on a lock-free union-find (a root is linked
// under a smaller root by compare-and-swap, so links never form a cycle).
int64_t find_components_par(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                            std::vector<int64_t> &comp) {
    std::unique_ptr<std::atomic<int64_t>[]> p(new std::atomic<int64_t>[n]);
    spx::parallel_ranges(n, 65536, [&](int64_t a, int64_t b) {
        for (int64_t i = a; i < b; i++) p[i].store(i, std::memory_order_relaxed);
    });
    auto find = [&](int64_t x) {
        for (;;) {
            int64_t px = p[x].load(std::memory_order_relaxed);
            if (px == x) return x;
            int64_t gx = p[px].load(std::memory_order_relaxed);
            if (gx != px) p[x].compare_exchange_weak(px, gx, std::memory_order_relaxed);
            x = gx;
        }
    };
    spx::parallel_ranges(n, 8192, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; c++)
            for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
                if (Ax[q] == 0.0) continue;
                int64_t a = Ai[q], b = c;
                for (;;) {
                    a = find(a);
                    b = find(b);
                    if (a == b) break;
                    if (a < b) std::swap(a, b);
                    int64_t expect = a;
                    if (p[a].compare_exchange_strong(expect, b, std::memory_order_relaxed)) break;
                }
            }
    });
    std::vector<int64_t> lab(n, -1);
    comp.assign(n, 0);
    int64_t nc = 0;
    for (int64_t i = 0; i < n; i++) {
        const int64_t r = find(i);
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

// stored entries from which the pattern checks run on side threads
constexpr int64_t kSideThreadsMin = 1 << 17;

// a side thread that is joined on every way out of its scope
struct SideThread {
    std::thread t;
    template <class F>
    void start(F &&f) { t = std::thread(std::forward<F>(f)); }
    void join() { if (t.joinable()) t.join(); }
    ~SideThread() { join(); }
};

int speigs_impl(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax, int64_t k,
                speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                double *lambda, double *V, double *resid, speigs_info *info,
                speigs_ext_info *einfo);

// Component split: rows grouped by component label, in row order.
struct CompSplit {
    int64_t ncomp = 0;
    std::vector<int64_t> sz, off, gidx, loc;
    void build(int64_t n, const std::vector<int64_t> &comp, int64_t nc) {
        ncomp = nc;
        sz.assign(nc, 0);
        off.assign(nc + 1, 0);
        gidx.resize(n);
        loc.resize(n);
        std::vector<int64_t> fill(nc, 0);
        for (int64_t i = 0; i < n; i++) sz[comp[i]]++;
        for (int64_t c = 0; c < nc; c++) off[c + 1] = off[c] + sz[c];
        for (int64_t i = 0; i < n; i++) {
            const int64_t c = comp[i], slot = off[c] + fill[c]++;
            gidx[slot] = i;
            loc[i] = slot - off[c];
        }
    }
};

// Result of one component's solve.
struct CompResult {
    int64_t kc = 0;
    std::vector<double> lam, res, vec;   // vec: nc x kc column-major (when wanted)
    speigs_info info;
    speigs_ext_info einfo;
};

// Solve every component with speigs_impl (which applies the reference's
// per-component routing: diagonal, dense or Krylov), kc = min(k, n_c).  The
// components are independent, so they are taken from a shared queue by a
// pool of host threads, largest first; each thread's solves run on their own
// CUDA streams and overlap on the GPU.  Returns 0 or the first error.
int solve_components(const int64_t *Ap, const int64_t *Ai, const double *Ax,
                     const std::vector<int64_t> &comp, const CompSplit &sp, int64_t k,
                     speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                     bool want_vec, std::vector<CompResult> &out) {
    const int64_t nc_all = sp.ncomp;
    out.assign(nc_all, CompResult());
    std::vector<int64_t> order(nc_all);
    for (int64_t c = 0; c < nc_all; c++) order[c] = c;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return sp.sz[a] > sp.sz[b]; });
    std::atomic<int64_t> next{0};
    std::atomic<int> err{0};
    auto worker = [&] {
        std::vector<int64_t> sAp, sAi;
        std::vector<double> sAx;
        for (;;) {
            const int64_t it = next.fetch_add(1);
            if (it >= nc_all || err.load() != 0) break;
            const int64_t ci = order[it], nc = sp.sz[ci];
            sAp.assign(nc + 1, 0);
            sAi.clear();
            sAx.clear();
            for (int64_t j = 0; j < nc; j++) {
                const int64_t gc = sp.gidx[sp.off[ci] + j];
                sAp[j] = (int64_t)sAi.size();
                for (int64_t q = Ap[gc]; q < Ap[gc + 1]; q++) {
                    const int64_t r = Ai[q];
                    if (comp[r] == ci) { sAi.push_back(sp.loc[r]); sAx.push_back(Ax[q]); }
                }
            }
            sAp[nc] = (int64_t)sAi.size();
            if (sAi.empty()) { sAi.push_back(0); sAx.push_back(0.0); }
            CompResult &R = out[ci];
            R.kc = std::min(k, nc);
            R.lam.assign(R.kc, 0.0);
            R.res.assign(R.kc, 0.0);
            if (want_vec) R.vec.assign((size_t)nc * R.kc, 0.0);
            const int rc = speigs_impl(nc, sAp.data(), sAi.data(), sAx.data(), R.kc, which, opts,
                                       ext, R.lam.data(), want_vec ? R.vec.data() : nullptr,
                                       R.res.data(), &R.info, &R.einfo);
            if (rc) {
                int expected = 0;
                err.compare_exchange_strong(expected, rc);
            }
        }
    };
    unsigned hw = std::thread::hardware_concurrency();
    int64_t nth = std::min<int64_t>(nc_all, std::max(1u, std::min(hw ? hw : 1u, 16u)));
    std::vector<std::thread> th;
    for (int64_t i = 1; i < nth; i++) th.emplace_back(worker);
    worker();
    for (auto &t : th) t.join();
    return err.load();
}

// Solve every component separately and merge by |lambda| (reference
// blocks_path, src/speigs_core.c:532-632).
int blocks_path(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax, int64_t k,
                speigs_which which, const speigs_opts *opts, const speigs_ext_opts *ext,
                const std::vector<int64_t> &comp, int64_t ncomp, double *lambda, double *V,
                double *resid, speigs_info *info, speigs_ext_info *einfo) {
    CompSplit sp;
    sp.build(n, comp, ncomp);
    std::vector<CompResult> cr;
    int rc = solve_components(Ap, Ai, Ax, comp, sp, k, which, opts, ext, V != nullptr, cr);
    if (rc) return rc;
    std::vector<double> clam, cres;
    std::vector<int64_t> ccomp, cslot;
    for (int64_t ci = 0; ci < ncomp; ci++) {
        const CompResult &R = cr[ci];
        if (einfo) {
            einfo->refine_steps += R.einfo.refine_steps;
            einfo->factor_solves += R.einfo.factor_solves;
            if (R.einfo.precision) einfo->precision = R.einfo.precision;
        }
        info->nops += R.info.nops;
        if (R.info.flag) info->flag = 1;
        for (int64_t t = 0; t < R.kc; t++) {
            clam.push_back(R.lam[t]);
            cres.push_back(R.res[t]);
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
        const int64_t i = ord[t].idx, ci = ccomp[i], sl = cslot[i], nc = sp.sz[ci];
        lambda[t] = clam[i];
        if (resid) resid[t] = cres[i];
        if (V) {
            memset(V + (size_t)t * n, 0, (size_t)n * sizeof(double));
            const double *src = cr[ci].vec.data() + (size_t)sl * nc;
            for (int64_t j = 0; j < nc; j++) V[(size_t)t * n + sp.gidx[sp.off[ci] + j]] = src[j];
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

int speigs_components(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                      const double *Ax, speigs_int *comp, speigs_int *ncomp) {
    if (n <= 0 || !Ap || !Ai || !Ax || !comp || !ncomp) return SPEIGS_ERR_ARG;
    std::vector<int64_t> c;
    *ncomp = Ap[n] >= kSideThreadsMin ? find_components_par(n, Ap, Ai, Ax, c)
                                      : find_components(n, Ap, Ai, Ax, c);
    memcpy(comp, c.data(), sizeof(int64_t) * (size_t)n);
    return SPEIGS_OK;
}

int speigs_batched(speigs_int n, const speigs_int *Ap, const speigs_int *Ai, const double *Ax,
                   speigs_int k, speigs_which which, const speigs_opts *opts,
                   const speigs_ext_opts *ext, const speigs_int *comp, speigs_int ncomp,
                   double *lambda, double *V, double *resid, speigs_int *nvals,
                   speigs_info *info) {
    speigs_opts defo;
    if (!opts) { speigs_default_opts(&defo); opts = &defo; }
    speigs_info li;
    if (!info) info = &li;
    memset(info, 0, sizeof *info);
    if (n <= 0 || !Ap || !Ai || !Ax || !lambda || !comp || ncomp <= 0 || k <= 0)
        return SPEIGS_ERR_ARG;
    for (int64_t i = 0; i < n; i++)
        if (comp[i] < 0 || comp[i] >= ncomp) return SPEIGS_ERR_ARG;
    if (opts->check_sym != 0 && check_symmetry(n, Ap, Ai, Ax) == 0) return SPEIGS_ERR_NOTSYM;
    std::vector<int64_t> cv(comp, comp + n);
    CompSplit sp;
    sp.build(n, cv, ncomp);
    for (int64_t c = 0; c < ncomp; c++)
        if (sp.sz[c] == 0) return SPEIGS_ERR_ARG;
    // the per-component calls repeat no symmetry check; only small
    // components take the dense route (the one-block dense eigensolver is
    // latency-bound beyond a few dozen rows), the rest the Krylov route
    speigs_opts o2 = *opts;
    o2.check_sym = 0;
    o2.dense_max = 64;
    std::vector<CompResult> cr;
    int rc = solve_components(Ap, Ai, Ax, cv, sp, k, which, &o2, ext, V != nullptr, cr);
    if (rc) return rc;
    memset(lambda, 0, sizeof(double) * (size_t)ncomp * k);
    if (resid) memset(resid, 0, sizeof(double) * (size_t)ncomp * k);
    if (V) memset(V, 0, sizeof(double) * (size_t)n * k);
    for (int64_t c = 0; c < ncomp; c++) {
        const CompResult &R = cr[c];
        for (int64_t t = 0; t < R.kc; t++) {
            lambda[c * k + t] = R.lam[t];
            if (resid) resid[c * k + t] = R.res[t];
            if (V) {
                const double *src = R.vec.data() + (size_t)t * sp.sz[c];
                for (int64_t j = 0; j < sp.sz[c]; j++) V[(size_t)t * n + sp.gidx[sp.off[c] + j]] = src[j];
            }
        }
        if (nvals) nvals[c] = R.kc;
        info->nops += R.info.nops;
        if (R.info.flag) info->flag = 1;
        info->nconv += R.info.nconv;
    }
    info->ncomp = ncomp;
    info->path = SPEIGS_PATH_BLOCKS;
    return SPEIGS_OK;
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
    const double tc = wall();
    // Large inputs: the symmetry check and the component labels run as
    // parallel passes, and the labels, the 1-norm and the CSR expansion side
    // by side; the route is taken in the reference's order.
    const bool par = Ap[n] >= kSideThreadsMin;
    bool full_sorted = false;
    if (opts->check_sym != 0) {
        const int sym = par ? check_symmetry_par(n, Ap, Ai, Ax, &full_sorted)
                            : check_symmetry(n, Ap, Ai, Ax);
        if (sym == 0) return SPEIGS_ERR_NOTSYM;
    }
    if (n == 1) {
        // a 1 x 1 matrix is its own eigenvalue: no numerical work to do
        double a = 0.0;
        for (int64_t p = Ap[0]; p < Ap[1]; p++) if (Ai[p] == 0) a = Ax[p];
        lambda[0] = a;
        if (V) V[0] = 1.0;
        if (resid) resid[0] = 0.0;
        info->nconv = 1;
        info->path = SPEIGS_PATH_DIAG;
        return SPEIGS_OK;
    }

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
    std::vector<int64_t> comp;
    int64_t ncomp = 1;
    SideThread comp_th;
    if (opts->detect) {
        if (par) comp_th.start([&] { ncomp = find_components_par(n, Ap, Ai, Ax, comp); });
        else ncomp = find_components(n, Ap, Ai, Ax, comp);
    }
    double anorm = 0.0;
    SideThread norm_th;
    if (par) norm_th.start([&] { anorm = norm1_upper(n, Ap, Ai, Ax); });
    else anorm = norm1_upper(n, Ap, Ai, Ax);
    HostCSR A;
    int rc = full_sorted ? spx::build_full_csr_sorted(n, Ap, Ai, Ax, &A)
                         : spx::build_full_csr(n, Ap, Ai, Ax, &A);
    comp_th.join();
    norm_th.join();
    if (anorm <= 0) anorm = 1.0;
    if (ncomp > 1) {
        spx::free_csr(&A);
        rc = blocks_path(n, Ap, Ai, Ax, k, which, opts, ext, comp, ncomp, lambda, V, resid, info,
                         einfo);
        info->t_iter = wall() - t0;
        return rc;
    }
    if (rc) return rc;
    info->anorm = anorm;
    const double t_checks = wall() - tc;
    // factor + Lanczos on the device; results come back sorted by |lambda|
    rc = spx::device_krylov(A, k, which, *opts, anorm, lambda, V, resid, info, nullptr, ext,
                            einfo);
    einfo->t_checks = t_checks;
    return rc;
}

}  // namespace
