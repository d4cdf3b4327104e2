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

// Phases of the calling thread's last speigs_batched (speigs_b200_batched_stats).
struct BatchedCallStats {
    double t_checks = 0, t_group = 0, t_seg = 0, t_rest = 0, t_total = 0;
    int64_t nkry = 0, nrest = 0, kry_rows = 0;
    spx::BatchedStats seg;
};
thread_local BatchedCallStats g_bstats;

// Symmetry verdict of the reference's input check (src/speigs_core.c:363-401):
// 1 when both triangles are stored and A equals its transpose entry for
// entry (values within 1e-12 relative), 2 when only the upper triangle is
// stored, 3 when only the lower, 0 otherwise.
//
// The reference builds the transpose by a counting sort, whose columns come
// out with nondecreasing row indices, and compares the two CSC arrays.  So,
// with both triangles stored, a column whose row indices decrease anywhere
// fails, and otherwise A equals its transpose exactly when every stored
// (r, c) -- the t-th entry of the run of row index r in column c -- meets,
// in column r, a run of row index c of the same length whose t-th value
// agrees.  Each column tests its own entries by binary search into the
// columns they mirror, so the columns are checked in parallel ranges.
// *full_sorted is set when the verdict is 1 and every column's row indices
// strictly increase (the layout build_full_csr_sorted expects).
int symmetry_verdict(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                     bool *full_sorted) {
    *full_sorted = false;
    std::atomic<int> up{0}, lo{0}, descending{0}, repeated{0}, outside{0};
    spx::parallel_ranges(n, 8192, [&](int64_t c0, int64_t c1) {
        bool u = false, l = false, dsc = false, rep = false, out = false;
        for (int64_t c = c0; c < c1; c++) {
            const int64_t *b = Ai + Ap[c], *e = Ai + Ap[c + 1];
            for (const int64_t *q = b; q < e; q++) {
                u |= *q < c;
                l |= *q > c;
                out |= *q < 0 || *q >= n;
                if (q > b) {
                    dsc |= q[0] < q[-1];
                    rep |= q[0] == q[-1];
                }
            }
        }
        if (u) up = 1;
        if (l) lo = 1;
        if (dsc) descending = 1;
        if (rep) repeated = 1;
        if (out) outside = 1;
    });
    if (!lo && up) return 2;
    if (!up && lo) return 3;
    if (!up && !lo) return 1;
    if (descending || outside) return 0;
    std::atomic<int> bad{0};
    spx::parallel_ranges(n, 8192, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1 && !bad.load(std::memory_order_relaxed); c++) {
            const int64_t *cb = Ai + Ap[c], *ce = Ai + Ap[c + 1];
            for (const int64_t *q = cb; q < ce; q++) {
                const int64_t r = *q;
                if (r == c) continue;   // a diagonal run mirrors itself
                const int64_t *mb = Ai + Ap[r], *me = Ai + Ap[r + 1];
                const int64_t *m0 = std::lower_bound(mb, me, c);
                int64_t t = 0, len_here = 1, len_there = 0;
                if (repeated) {
                    // position within this column's run of r, and both run lengths
                    const auto run = std::equal_range(cb, ce, r);
                    t = q - run.first;
                    len_here = run.second - run.first;
                    len_there = std::upper_bound(m0, me, c) - m0;
                } else {
                    len_there = (m0 != me && *m0 == c) ? 1 : 0;
                }
                if (len_there != len_here) { bad = 1; break; }
                const double a = Ax[q - Ai], m = Ax[(m0 - Ai) + t];
                const double big = std::max(fabs(a), fabs(m));
                if (fabs(a - m) > 1e-12 * (big > 0 ? big : 1.0)) { bad = 1; break; }
            }
        }
    });
    if (bad) return 0;
    *full_sorted = !repeated;
    return 1;
}

// The reference's diagonal gate (src/speigs_core.c:801): no stored entry
// off the diagonal, whatever its value.
bool pattern_is_diagonal(int64_t n, const int64_t *Ap, const int64_t *Ai) {
    std::atomic<int> off{0};
    spx::parallel_ranges(n, 1 << 16, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1 && !off.load(std::memory_order_relaxed); c++)
            if (std::any_of(Ai + Ap[c], Ai + Ap[c + 1], [c](int64_t r) { return r != c; }))
                off = 1;
    });
    return !off;
}

// Connected components over the numerically nonzero stored entries, labelled
// 0, 1, ... in the order in which each component's first row appears -- the
// split the reference makes (find_components, src/speigs_core.c:445-466).
// The unions run in parallel ranges of columns on a lock-free union-find: a
// root is linked under a smaller root by compare-and-swap, so links never
// form a cycle, and finds halve their paths as they go.
int64_t find_components(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
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
    // roots are the smallest row of their component, so a component's label
    // is fixed when its root is reached in row order
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

// The reference's banded-route gate (src/speigs_core.c:865-893), decided on
// the caller's CSC pattern: a reverse Cuthill-McKee order (breadth-first
// levels from the lowest-degree unvisited vertex, each vertex's unvisited
// neighbours appended in order of increasing column count, ties kept in
// storage order, the whole order reversed), the bandwidth kd of A under it,
// and the band's size and occupancy: kd <= band_max (512 when 0), (kd + 1) n
// <= 2e7 cells and nnz / (n kd) >= 0.05.
bool banded_gate(int64_t n, const int64_t *Ap, const int64_t *Ai, const speigs_opts &o) {
    const int64_t bmax = o.band_max ? o.band_max : 512;
    if (bmax <= 0) return false;
    std::vector<int64_t> order;
    order.reserve(n);
    std::vector<char> seen(n, 0);
    auto degree = [&](int64_t v) { return Ap[v + 1] - Ap[v]; };
    std::vector<int64_t> fresh;
    int64_t scan = 0;
    while ((int64_t)order.size() < n) {
        while (seen[scan]) scan++;
        // the lowest-degree unvisited vertex at or after the first unvisited one
        int64_t s = scan;
        for (int64_t i = scan; i < n; i++)
            if (!seen[i] && degree(i) < degree(s)) s = i;
        seen[s] = 1;
        size_t head = order.size();
        order.push_back(s);
        while (head < order.size()) {
            const int64_t v = order[head++];
            fresh.clear();
            for (int64_t q = Ap[v]; q < Ap[v + 1]; q++) {
                const int64_t w = Ai[q];
                if (w < 0 || w >= n) return false;
                if (!seen[w]) { seen[w] = 1; fresh.push_back(w); }
            }
            std::stable_sort(fresh.begin(), fresh.end(),
                             [&](int64_t a, int64_t b) { return degree(a) < degree(b); });
            order.insert(order.end(), fresh.begin(), fresh.end());
        }
    }
    // position of each vertex in the reversed order
    std::vector<int64_t> pos(n);
    for (int64_t i = 0; i < n; i++) pos[order[n - 1 - i]] = i;
    int64_t kd = 0;
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++)
            kd = std::max<int64_t>(kd, std::llabs(pos[Ai[q]] - pos[c]));
    const double cells = (double)(kd + 1) * (double)n;
    const double occupancy = kd > 0 ? (double)Ap[n] / ((double)n * (double)kd) : 1.0;
    return kd <= bmax && cells <= 2.0e7 && occupancy >= 0.05;
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
                     bool want_vec, std::vector<CompResult> &out,
                     const std::vector<int64_t> *subset = nullptr) {
    if ((int64_t)out.size() != sp.ncomp) out.assign(sp.ncomp, CompResult());
    std::vector<int64_t> order;
    if (subset) {
        order = *subset;
    } else {
        order.resize(sp.ncomp);
        for (int64_t c = 0; c < sp.ncomp; c++) order[c] = c;
    }
    const int64_t nc_all = (int64_t)order.size();
    if (nc_all == 0) return 0;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return sp.sz[a] > sp.sz[b]; });
    std::atomic<int> err{0};
    // the caller's device: worker threads start on device 0 and adopt it
    const int dev = spx::current_device();
    auto solve_one = [&](int64_t it) {
        const int64_t ci = order[it], nc = sp.sz[ci];
        std::vector<int64_t> tAp(nc + 1, 0), tAi;
        std::vector<double> tAx;
        for (int64_t j = 0; j < nc; j++) {
            const int64_t gc = sp.gidx[sp.off[ci] + j];
            tAp[j] = (int64_t)tAi.size();
            for (int64_t q = Ap[gc]; q < Ap[gc + 1]; q++) {
                const int64_t r = Ai[q];
                if (comp[r] == ci) { tAi.push_back(sp.loc[r]); tAx.push_back(Ax[q]); }
            }
        }
        tAp[nc] = (int64_t)tAi.size();
        if (tAi.empty()) { tAi.push_back(0); tAx.push_back(0.0); }
        CompResult &R = out[ci];
        R.kc = std::min(k, nc);
        R.lam.assign(R.kc, 0.0);
        R.res.assign(R.kc, 0.0);
        if (want_vec) R.vec.assign((size_t)nc * R.kc, 0.0);
        const int rc = speigs_impl(nc, tAp.data(), tAi.data(), tAx.data(), R.kc, which, opts,
                                   ext, R.lam.data(), want_vec ? R.vec.data() : nullptr,
                                   R.res.data(), &R.info, &R.einfo);
        if (rc) {
            int expected = 0;
            err.compare_exchange_strong(expected, rc);
        }
    };
    unsigned hw = std::thread::hardware_concurrency();
    const int nth = (int)std::min<int64_t>(nc_all, std::max(1u, std::min(hw ? hw : 1u, 16u)));
    spx::run_pool(nc_all, nth, [dev] { spx::use_device(dev); }, solve_one,
                  [&] { return err.load() != 0; });
    return err.load();
}

// The components in `kry` (Krylov route, each connected and larger than the
// dense gate) solved together by the segmented lockstep Lanczos: their rows
// become contiguous segments, largest component first, of one
// block-diagonal matrix whose full CSR is built from the upper triangle as
// for a single call.  Results land in out[c] as solve_components leaves
// them (sorted by |lambda|, vectors on the component's rows).  Returns 0, a
// negative code, or 1 when these components must be solved one by one.
// Components still iterating when few remain are appended to *handed_out,
// to be solved one by one (the lockstep step solves the whole forest).
int batched_krylov(const int64_t *Ap, const int64_t *Ai, const double *Ax,
                   const std::vector<int64_t> &comp, const CompSplit &sp,
                   std::vector<int64_t> kry, int64_t k, speigs_which which,
                   const speigs_opts &o, bool want_vec, std::vector<CompResult> &out,
                   std::vector<int64_t> *handed_out, int handoff, bool full_sorted) {
    const double t_group0 = wall();
    std::stable_sort(kry.begin(), kry.end(),
                     [&](int64_t a, int64_t b) { return sp.sz[a] > sp.sz[b]; });
    const int nseg = (int)kry.size();
    std::vector<int32_t> off(nseg + 1, 0);
    for (int q = 0; q < nseg; q++) off[q + 1] = off[q] + (int32_t)sp.sz[kry[q]];
    const int64_t ng = off[nseg];
    // group CSC: segment q's column jl is the component's jl-th row (original
    // order).  Segments are independent: their column counts, entries and
    // norms are built by a pool of host threads (largest segments first),
    // with the offsets from a prefix sum in between.
    std::vector<int64_t> Gp(ng + 1, 0);
    std::vector<double> anorm(nseg, 0.0);
    const int nth = (int)std::min<int64_t>(spx::host_threads(), nseg);
    auto over_segments = [&](auto &&body) {
        std::atomic<int> next{0};
        auto worker = [&] {
            for (int q; (q = next.fetch_add(1)) < nseg;) body(q);
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nth; t++) th.emplace_back(worker);
        worker();
        for (auto &t : th) t.join();
    };
    over_segments([&](int q) {
        const int64_t c = kry[q], nc = sp.sz[c];
        for (int64_t jl = 0; jl < nc; jl++) {
            const int64_t gc = sp.gidx[sp.off[c] + jl];
            int64_t cnt = 0;
            for (int64_t e = Ap[gc]; e < Ap[gc + 1]; e++) cnt += comp[Ai[e]] == c;
            Gp[off[q] + jl + 1] = cnt;
        }
    });
    for (int64_t g = 0; g < ng; g++) Gp[g + 1] += Gp[g];
    std::vector<int64_t> Gi((size_t)Gp[ng]);
    std::vector<double> Gx((size_t)Gp[ng]);
    over_segments([&](int q) {
        const int64_t c = kry[q], nc = sp.sz[c];
        std::vector<double> colsum(nc, 0.0);
        for (int64_t jl = 0; jl < nc; jl++) {
            const int64_t g = off[q] + jl, gc = sp.gidx[sp.off[c] + jl];
            int64_t d = Gp[g];
            for (int64_t e = Ap[gc]; e < Ap[gc + 1]; e++) {
                const int64_t r = Ai[e];
                if (comp[r] != c) continue;
                const int64_t rl = sp.loc[r];
                Gi[d] = off[q] + rl;
                Gx[d++] = Ax[e];
                // ||A_c||_1 of the symmetric matrix of the upper triangle
                if (rl <= jl) {
                    colsum[jl] += fabs(Ax[e]);
                    if (rl != jl) colsum[rl] += fabs(Ax[e]);
                }
            }
        }
        double mx = 0.0;
        for (double v : colsum) mx = std::max(mx, v);
        anorm[q] = mx > 0 ? mx : 1.0;
    });
    HostCSR A;
    // a full, sorted symmetric input keeps both properties in its diagonal
    // blocks (each component's rows keep their order)
    int rc = full_sorted ? spx::build_full_csr_sorted(ng, Gp.data(), Gi.data(), Gx.data(), &A)
                         : spx::build_full_csr(ng, Gp.data(), Gi.data(), Gx.data(), &A);
    if (rc) return rc;
    std::vector<double> lam((size_t)nseg * k), res((size_t)nseg * k);
    std::vector<double> X(want_vec ? (size_t)ng * k : 0);
    std::vector<int64_t> nconv(nseg), nops(nseg), rst(nseg);
    std::vector<int> flag(nseg);
    spx::BatchedStats &bst = g_bstats.seg;
    bst = spx::BatchedStats();
    g_bstats.kry_rows = ng;
    g_bstats.t_group = wall() - t_group0;
    std::vector<int> handed(nseg, 0);
    rc = spx::device_batched_krylov(A, nseg, off.data(), k, which, o, anorm.data(), lam.data(),
                                    res.data(), want_vec ? X.data() : nullptr, nconv.data(),
                                    nops.data(), rst.data(), flag.data(), &bst,
                                    handed_out ? handed.data() : nullptr, handoff);
    if (rc) return rc;
    for (int q = 0; q < nseg; q++) {
        const int64_t c = kry[q], nc = sp.sz[c];
        if (handed[q]) {
            handed_out->push_back(c);
            continue;
        }
        CompResult &R = out[c];
        R.kc = std::min(k, nc);
        // sort by |lambda| as speigs() does: ascending 'sm', descending 'lm'
        std::vector<int64_t> idx(R.kc);
        for (int64_t t = 0; t < R.kc; t++) idx[t] = t;
        const double *lq = lam.data() + (size_t)q * k;
        std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
            return which == SPEIGS_SM ? fabs(lq[a]) < fabs(lq[b]) : fabs(lq[a]) > fabs(lq[b]);
        });
        R.lam.assign(R.kc, 0.0);
        R.res.assign(R.kc, 0.0);
        if (want_vec) R.vec.assign((size_t)nc * R.kc, 0.0);
        for (int64_t t = 0; t < R.kc; t++) {
            R.lam[t] = lq[idx[t]];
            R.res[t] = res[(size_t)q * k + idx[t]];
            if (want_vec)
                memcpy(R.vec.data() + (size_t)t * nc, X.data() + (size_t)idx[t] * ng + off[q],
                       sizeof(double) * nc);
        }
        memset(&R.info, 0, sizeof R.info);
        R.info.nconv = nconv[q];
        R.info.nops = nops[q];
        R.info.restarts = rst[q];
        R.info.flag = flag[q];
        R.info.anorm = anorm[q];
        R.info.path = which == SPEIGS_SM ? SPEIGS_PATH_SHIFTINV : SPEIGS_PATH_DIRECT;
        memset(&R.einfo, 0, sizeof R.einfo);
    }
    return 0;
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
    bool full_sorted = false;
    return symmetry_verdict(n, Ap, Ai, Ax, &full_sorted);
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
    *ncomp = find_components(n, Ap, Ai, Ax, c);
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
    g_bstats = BatchedCallStats();
    const double t0 = wall();
    if (n <= 0 || !Ap || !Ai || !Ax || !lambda || !comp || ncomp <= 0 || k <= 0)
        return SPEIGS_ERR_ARG;
    for (int64_t i = 0; i < n; i++)
        if (comp[i] < 0 || comp[i] >= ncomp) return SPEIGS_ERR_ARG;
    bool full_sorted = false;
    if (opts->check_sym != 0 && symmetry_verdict(n, Ap, Ai, Ax, &full_sorted) == 0)
        return SPEIGS_ERR_NOTSYM;
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
    std::vector<CompResult> cr(ncomp);
    // Components that take the Krylov route (larger than the dense gate) are
    // solved together in lockstep by the segmented Lanczos; the others, and
    // all of them when the forest needs a shift or an extension option asks
    // for another operator, one per host thread.
    std::vector<int64_t> kry, rest;
    const bool seg_ok = !ext || (ext->precision == SPEIGS_B200_FP64 && !ext->warm && ext->block <= 0);
    for (int64_t c = 0; c < ncomp; c++) {
        const int64_t nc = sp.sz[c];
        const bool dense = nc <= o2.dense_max || 4 * k > nc;
        if (seg_ok && nc > 1 && !dense) kry.push_back(c);
        else rest.push_back(c);
    }
    g_bstats.t_checks = wall() - t0;
    g_bstats.nkry = (int64_t)kry.size();
    if (!kry.empty()) {
        const double ts = wall();
        std::vector<int64_t> handed;
        const int handoff = !ext || ext->handoff == 0 ? 8 : ext->handoff;
        int rcs = batched_krylov(Ap, Ai, Ax, cv, sp, kry, k, which, o2, V != nullptr, cr, &handed,
                                 handoff, full_sorted);
        if (rcs < 0) return rcs;
        if (rcs == 1) rest.insert(rest.end(), kry.begin(), kry.end());
        else rest.insert(rest.end(), handed.begin(), handed.end());
        g_bstats.t_seg = wall() - ts - g_bstats.t_group;
    }
    g_bstats.nrest = (int64_t)rest.size();
    const double tr = wall();
    int rc = solve_components(Ap, Ai, Ax, cv, sp, k, which, &o2, ext, V != nullptr, cr, &rest);
    g_bstats.t_rest = wall() - tr;
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
    g_bstats.t_total = wall() - t0;
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
        const int sym = symmetry_verdict(n, Ap, Ai, Ax, &full_sorted);
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
    if (opts->detect && pattern_is_diagonal(n, Ap, Ai)) {
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
        if (par) comp_th.start([&] { ncomp = find_components(n, Ap, Ai, Ax, comp); });
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
    // the reference's banded route ('sm'): the band is factored on the device
    // by dissecting it into independent segments (the supernodal factor under
    // nested dissection), with the same shift escalation
    const bool banded = which == SPEIGS_SM && banded_gate(n, Ap, Ai, *opts);
    // factor + Lanczos on the device; results come back sorted by |lambda|
    rc = spx::device_krylov(A, k, which, *opts, anorm, lambda, V, resid, info, nullptr, ext,
                            einfo, banded);
    einfo->t_checks = t_checks;
    return rc;
}

}  // namespace

int speigs_b200_batched_stats(double *times, int64_t *counts) {
    if (!times || !counts) return SPEIGS_ERR_ARG;
    const BatchedCallStats &b = g_bstats;
    const double t[9] = {b.t_checks, b.t_group, b.seg.t_analyze, b.seg.t_factor, b.seg.t_iter,
                         b.t_seg, b.t_rest, b.t_total, b.seg.t_total};
    const int64_t c[7] = {b.nkry, b.nrest, b.seg.handed, b.seg.steps, b.seg.cycles, b.kry_rows,
                          b.seg.graph ? 1 : 0};
    memcpy(times, t, sizeof t);
    memcpy(counts, c, sizeof c);
    return SPEIGS_OK;
}
