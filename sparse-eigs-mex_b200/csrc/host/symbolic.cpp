// Host symbolic analysis: ordering, elimination tree, column counts,
// supernodes, row structures, relative maps, tree levels.
//
// This is the project's own replacement for the analysis that
// cholmod_l_analyze performs in the reference (src/speigs_core.c:934, with
// the ordering choice at :859-863).  The numeric work it prepares runs on the
// device.
#include "symbolic.h"
#include "parallel.h"

#include <algorithm>
#include <mutex>
#include <functional>
#include <map>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

namespace {

struct Graph {
    int32_t n;
    const int64_t *rp;
    const int32_t *ci;
};

// ---------------------------------------------------------------- ordering --

// Exact minimum degree on a region of at most 64 vertices, using bitset
// adjacency of the elimination graph.  Appends the elimination order.
void leaf_mindeg(const Graph &g, const std::vector<int32_t> &verts,
                 std::vector<int32_t> &local, int32_t *out) {
    const int m = (int)verts.size();
    for (int a = 0; a < m; a++) local[verts[a]] = a;
    uint64_t adj[64];
    for (int a = 0; a < m; a++) {
        uint64_t bits = 0;
        int32_t v = verts[a];
        for (int64_t p = g.rp[v]; p < g.rp[v + 1]; p++) {
            int32_t u = g.ci[p];
            int32_t b = local[u];
            if (u != v && b >= 0 && b < m && verts[b] == u) bits |= (1ull << b);
        }
        adj[a] = bits;
    }
    uint64_t alive = (m == 64) ? ~0ull : ((1ull << m) - 1);
    for (int t = 0; t < m; t++) {
        int best = -1, bd = 1 << 30;
        for (int a = 0; a < m; a++) {
            if (!((alive >> a) & 1)) continue;
            int d = __builtin_popcountll(adj[a] & alive);
            if (d < bd) { bd = d; best = a; }
        }
        out[t] = verts[best];
        uint64_t nb = adj[best] & alive & ~(1ull << best);
        uint64_t it = nb;
        while (it) {
            int b = __builtin_ctzll(it);
            it &= it - 1;
            adj[b] |= nb & ~(1ull << b);
        }
        alive &= ~(1ull << best);
    }
    for (int a = 0; a < m; a++) local[verts[a]] = -1;
}

// Regions are ordered recursively; the two halves of a split touch disjoint
// vertex sets (a separator leaves no edge between them), so large halves are
// ordered on separate threads.  The per-vertex arrays are shared: a region
// only writes the entries of its own vertices and reads those of its
// neighbours, which lie in the region itself or in separators that are
// already final.
struct NDState {
    const Graph &g;
    // region id and BFS level scratch of every vertex, side by side: a BFS
    // step reads both for each neighbour
    struct PartLevel { int32_t part, level; };
    std::vector<PartLevel> pl;
    std::vector<int32_t> local;  // leaf-local index scratch
    std::atomic<int32_t> next_id{1};
    std::atomic<int> spare_threads{0};
    // Independent ranges of the ordering, for the elimination tree: a
    // region [lo, lo + m) of at least kRecordMin vertices whose columns
    // split into child ranges that reach only themselves and later columns
    // (the halves of a separation, or the connected pieces of a region),
    // followed by the columns of the separator (none for pieces).
    struct Split {
        int32_t lo, m;
        std::vector<std::pair<int32_t, int32_t>> parts;   // (first, count)
    };
    std::mutex split_mu;
    std::vector<Split> splits;
    static constexpr int32_t kRecordMin = 8192;
    void record(Split &&sp) {
        std::lock_guard<std::mutex> lk(split_mu);
        splits.push_back(std::move(sp));
    }
    int32_t *perm;
    explicit NDState(const Graph &gg, int32_t *p)
        : g(gg), pl(gg.n, PartLevel{0, -1}), local(gg.n, -1), perm(p) {}

    // BFS inside region `id` from `src`; fills queue[0..cnt), pl[].level; returns
    // the number reached and the eccentricity in *depth.  `queue` holds at
    // least as many entries as the region has vertices.
    int32_t bfs(int32_t id, int32_t src, int32_t *depth, std::vector<int32_t> &queue) {
        int32_t head = 0, tail = 0;
        queue[tail++] = src;
        pl[src].level = 0;
        int32_t d = 0;
        while (head < tail) {
            int32_t v = queue[head++];
            int32_t lv = pl[v].level;
            if (lv > d) d = lv;
            for (int64_t p = g.rp[v]; p < g.rp[v + 1]; p++) {
                int32_t u = g.ci[p];
                if (pl[u].part == id && pl[u].level < 0) {
                    pl[u].level = lv + 1;
                    queue[tail++] = u;
                }
            }
        }
        *depth = d;
        return tail;
    }
    void clear_levels(const std::vector<int32_t> &queue, int32_t cnt) {
        for (int32_t i = 0; i < cnt; i++) pl[queue[i]].level = -1;
    }
    int32_t degree_in(int32_t v, int32_t id) const {
        int32_t d = 0;
        for (int64_t p = g.rp[v]; p < g.rp[v + 1]; p++)
            if (pl[g.ci[p]].part == id) d++;
        return d;
    }

    // Order the vertices `verts` (all carrying region id `id`) into
    // perm[lo .. lo+|verts|).  `hint` (or -1) is a vertex of the region that
    // was peripheral in the parent's level structure: the start of the
    // parent's BFS for the near half, its deepest vertex for the far half.
    void order_region(std::vector<int32_t> verts, int32_t id, int32_t lo, int32_t hint = -1) {
        const int32_t m = (int32_t)verts.size();
        if (m == 0) return;
        if (m <= 64) {
            leaf_mindeg(g, verts, local, perm + lo);
            return;
        }
        std::vector<int32_t> queue(m);
        // pseudo-peripheral start: the hint, else the lowest degree vertex;
        // then repeated BFS from the deepest level
        int32_t src = hint;
        if (src < 0 || pl[src].part != id) {
            src = verts[0];
            int32_t bestdeg = degree_in(verts[0], id);
            for (int32_t v : verts) {
                int32_t d = degree_in(v, id);
                if (d < bestdeg) { bestdeg = d; src = v; }
            }
        }
        int32_t depth = 0, cnt = bfs(id, src, &depth, queue);
        if (cnt < m) {
            // disconnected region: order each connected piece on its own
            std::vector<std::vector<int32_t>> pieces;
            std::vector<int32_t> ids;
            pieces.emplace_back(queue.begin(), queue.begin() + cnt);
            clear_levels(queue, cnt);
            ids.push_back(next_id++);
            for (int32_t v : pieces[0]) pl[v].part = ids[0];
            for (int32_t v : verts) {
                if (pl[v].part != id) continue;
                int32_t d2 = 0, c2 = bfs(id, v, &d2, queue);
                pieces.emplace_back(queue.begin(), queue.begin() + c2);
                clear_levels(queue, c2);
                ids.push_back(next_id++);
                for (int32_t u : pieces.back()) pl[u].part = ids.back();
            }
            verts.clear();
            verts.shrink_to_fit();
            if (m >= kRecordMin) {
                Split sp{lo, m, {}};
                int32_t at2 = lo;
                for (auto &pc : pieces) {
                    sp.parts.push_back({at2, (int32_t)pc.size()});
                    at2 += (int32_t)pc.size();
                }
                record(std::move(sp));
            }
            // the pieces touch disjoint vertex sets: with spare threads they
            // are ordered concurrently, largest first, each into its own
            // range of perm (the result does not depend on the schedule)
            std::vector<int32_t> at(pieces.size());
            int32_t a0 = lo;
            for (size_t i = 0; i < pieces.size(); i++) {
                at[i] = a0;
                a0 += (int32_t)pieces[i].size();
            }
            const int avail = m >= kParallelMin && pieces.size() > 1
                                  ? std::max(0, spare_threads.exchange(0)) : 0;
            const int nw = (int)std::min<size_t>(pieces.size(), (size_t)avail + 1);
            if (nw > 1) {
                std::vector<int32_t> big(pieces.size());
                for (size_t i = 0; i < pieces.size(); i++) big[i] = (int32_t)i;
                std::stable_sort(big.begin(), big.end(), [&](int32_t x, int32_t y) {
                    return pieces[x].size() > pieces[y].size();
                });
                std::atomic<size_t> nexti{0};
                auto work = [&] {
                    for (size_t q; (q = nexti.fetch_add(1)) < big.size();) {
                        const int32_t i = big[q];
                        order_region(std::move(pieces[i]), ids[i], at[i]);
                    }
                };
                std::vector<std::thread> th;
                for (int t = 1; t < nw; t++) th.emplace_back(work);
                work();
                for (auto &t : th) t.join();
            } else {
                for (size_t i = 0; i < pieces.size(); i++)
                    order_region(std::move(pieces[i]), ids[i], at[i]);
            }
            spare_threads.fetch_add(avail);
            return;
        }
        for (int it = 0; it < 6; it++) {
            // candidate: min-degree vertex in the last level
            int32_t cand = -1, cd = 1 << 30;
            for (int32_t i = cnt - 1; i >= 0 && pl[queue[i]].level == depth; i--) {
                int32_t d = degree_in(queue[i], id);
                if (d < cd) { cd = d; cand = queue[i]; }
            }
            clear_levels(queue, cnt);
            int32_t d2 = 0;
            bfs(id, cand, &d2, queue);
            if (d2 < depth) {
                // shallower: redo the BFS from src to keep its levels
                clear_levels(queue, cnt);
                bfs(id, src, &depth, queue);
                break;
            }
            src = cand;
            if (d2 == depth) break;  // as deep: keep the candidate's levels
            depth = d2;
        }
        if (depth < 2) {
            // too shallow to split (clique-like): order by degree, low first
            std::vector<int32_t> vv(queue.begin(), queue.begin() + cnt);
            clear_levels(queue, cnt);
            std::stable_sort(vv.begin(), vv.end(), [&](int32_t a, int32_t b) {
                return degree_in(a, id) < degree_in(b, id);
            });
            for (int32_t i = 0; i < m; i++) perm[lo + i] = vv[i];
            return;
        }
        // level sizes
        std::vector<int32_t> lsz(depth + 1, 0);
        for (int32_t i = 0; i < cnt; i++) lsz[pl[queue[i]].level]++;
        std::vector<int64_t> cum(depth + 2, 0);
        for (int32_t l = 0; l <= depth; l++) cum[l + 1] = cum[l] + lsz[l];
        // choose separator level: smallest level subject to balance.  The
        // larger half is ordered after the split on the critical path, so the
        // bound (at least 35 % on the smaller side) also keeps the recursion
        // short: on 3-D grids it gives ~5 % fewer factor flops than 30 % at
        // about the same fill, and a shorter ordering.
        int32_t best = -1;
        double bestscore = 1e300;
        for (int32_t l = 1; l < depth; l++) {
            int64_t a = cum[l], b = (int64_t)m - cum[l + 1];
            double bal = (double)std::min(a, b) / (double)(a + b);
            if (bal < 0.35) continue;
            double score = (double)lsz[l] * (1.0 + 0.5 * (0.5 - bal));
            if (score < bestscore) { bestscore = score; best = l; }
        }
        if (best < 0) {
            // take the median level
            for (int32_t l = 1; l < depth; l++)
                if (2 * cum[l + 1] >= m) { best = l; break; }
            if (best < 0) best = depth / 2;
        }
        const int32_t ida = next_id++, idb = next_id++, ids = next_id++;
        // peripheral vertices of the two halves: the BFS start (level 0) and
        // the last vertex reached (level `depth`)
        const int32_t hint_a = src, hint_b = queue[cnt - 1];
        std::vector<int32_t> A, B, Sp;
        for (int32_t i = 0; i < cnt; i++) {
            int32_t v = queue[i], l = pl[v].level;
            if (l < best) { pl[v].part = ida; }
            else if (l > best) { pl[v].part = idb; }
            else { pl[v].part = ids; }
        }
        clear_levels(queue, cnt);
        // thin the separator: a separator vertex with no neighbour on one side
        // can join the other side.
        for (int32_t v : verts) {
            if (pl[v].part != ids) continue;
            bool hasA = false, hasB = false;
            for (int64_t p = g.rp[v]; p < g.rp[v + 1]; p++) {
                int32_t u = g.ci[p];
                if (pl[u].part == ida) hasA = true;
                else if (pl[u].part == idb) hasB = true;
            }
            if (!hasB) pl[v].part = ida;
            else if (!hasA) pl[v].part = idb;
        }
        for (int32_t v : verts) {
            if (pl[v].part == ida) A.push_back(v);
            else if (pl[v].part == idb) B.push_back(v);
            else Sp.push_back(v);
        }
        const int32_t na = (int32_t)A.size(), nb = (int32_t)B.size();
        if (m >= kRecordMin) record(Split{lo, m, {{lo, na}, {lo + na, nb}}});
        // separator last, ordered by minimum degree when small
        if ((int32_t)Sp.size() <= 64) {
            leaf_mindeg(g, Sp, local, perm + lo + na + nb);
        } else {
            for (int32_t i = 0; i < (int32_t)Sp.size(); i++) perm[lo + na + nb + i] = Sp[i];
        }
        verts.clear();
        verts.shrink_to_fit();
        queue.clear();
        queue.shrink_to_fit();
        if (na > kParallelMin && nb > kParallelMin && spare_threads.fetch_sub(1) > 0) {
            // the helper returns its slot as soon as its half is done
            std::thread t([this, &A, ida, lo, hint_a] {
                order_region(std::move(A), ida, lo, hint_a);
                spare_threads.fetch_add(1);
            });
            order_region(std::move(B), idb, lo + na, hint_b);
            t.join();
        } else {
            if (na > kParallelMin && nb > kParallelMin) spare_threads.fetch_add(1);
            order_region(std::move(A), ida, lo, hint_a);
            order_region(std::move(B), idb, lo + na, hint_b);
        }
    }
    static constexpr int32_t kParallelMin = 4096;
};

}  // namespace

namespace {
using Splits = std::vector<NDState::Split>;

int order_nd(int32_t n, const int64_t *rowptr, const int32_t *col, int32_t *perm,
             Splits *splits) {
    if (n <= 0 || !rowptr || !col || !perm) return -1;
    try {
        Graph g{n, rowptr, col};
        NDState st(g, perm);
        const unsigned hw = std::thread::hardware_concurrency();
        // helper threads for the halves of a split: more than the cores, so
        // that a large half never waits behind its sibling's whole subtree
        // because every helper was taken at the moment of its split (the
        // ordering itself does not depend on the schedule)
        st.spare_threads = (int)std::min(hw > 1 ? 4 * hw : 0u, 64u);
        std::vector<int32_t> all(n);
        for (int32_t i = 0; i < n; i++) all[i] = i;
        st.order_region(std::move(all), 0, 0);
        if (splits) splits->swap(st.splits);
    } catch (const std::bad_alloc &) {
        return -2;
    }
    return 0;
}
}  // namespace

extern "C" int spx_order(int32_t n, const int64_t *rowptr, const int32_t *col,
                         int ordering, int32_t *perm) {
    (void)ordering;  // nested dissection for every size; leaves by minimum degree
    return order_nd(n, rowptr, col, perm, nullptr);
}

namespace {

// cs-style leaf test of Gilbert, Ng and Peyton's column-count algorithm.
inline int32_t gnp_leaf(int32_t i, int32_t j, const int32_t *first, int32_t *maxfirst,
                        int32_t *prevleaf, int32_t *ancestor, int *jleaf) {
    *jleaf = 0;
    if (i <= j || first[j] <= maxfirst[i]) return -1;
    maxfirst[i] = first[j];
    int32_t jprev = prevleaf[i];
    prevleaf[i] = j;
    *jleaf = (jprev == -1) ? 1 : 2;
    if (*jleaf == 1) return i;
    int32_t q = jprev;
    while (q != ancestor[q]) q = ancestor[q];
    for (int32_t s = jprev, sp; s != q; s = sp) {
        sp = ancestor[s];
        ancestor[s] = q;
    }
    return q;
}

}  // namespace

extern "C" void spx_symbolic_free(spx_symbolic *S) {
    if (!S) return;
    free(S->perm); free(S->iperm); free(S->sfirst); free(S->sparent);
    free(S->rowptr); free(S->rows); free(S->relmap); free(S->frontptr);
    free(S->col2sup); free(S->level_ptr); free(S->level_sup);
    free(S->child_ptr); free(S->child_list);
    memset(S, 0, sizeof *S);
}

// items per host thread below which a pass stays on one thread
constexpr int64_t kGrain = 16384;

template <class T>
static T *xalloc(size_t cnt) {
    T *p = (T *)malloc((cnt ? cnt : 1) * sizeof(T));
    if (!p) throw std::bad_alloc();
    return p;
}

extern "C" int spx_analyze(int32_t n, const int64_t *rowptr, const int32_t *col,
                           int ordering, spx_symbolic *S) {
    if (!S || n <= 0 || !rowptr || !col) return -1;
    memset(S, 0, sizeof *S);
    try {
        S->n = n;
        // ---- 1. ordering
        std::vector<int32_t> perm0(n);
        Splits splits;
        (void)ordering;  // nested dissection for every size; leaves by minimum degree
        int rc = order_nd(n, rowptr, col, perm0.data(), &splits);
        if (rc) return rc;
        std::vector<int32_t> ip0(n);
        for (int32_t i = 0; i < n; i++) ip0[perm0[i]] = i;

        // ---- 2. permuted adjacency (new numbering), without the diagonal
        std::vector<int64_t> prp(n + 1, 0);
        spx::parallel_ranges(n, kGrain, [&](int64_t lo, int64_t hi) {
            for (int64_t j = lo; j < hi; j++) {
                const int32_t o = perm0[j];
                int64_t c = 0;
                for (int64_t p = rowptr[o]; p < rowptr[o + 1]; p++) c += (col[p] != o);
                prp[j + 1] = c;
            }
        });
        for (int32_t j = 0; j < n; j++) prp[j + 1] += prp[j];
        std::vector<int32_t> pci(prp[n]);
        spx::parallel_ranges(n, kGrain, [&](int64_t lo, int64_t hi) {
            for (int64_t j = lo; j < hi; j++) {
                const int32_t o = perm0[j];
                int64_t q = prp[j];
                for (int64_t p = rowptr[o]; p < rowptr[o + 1]; p++)
                    if (col[p] != o) pci[q++] = ip0[col[p]];
            }
        });

        // ---- 3. elimination tree (Liu, with path compression)
        // The columns of each part of a recorded split reach, below
        // themselves, only their own part, and Liu's walks from them stay
        // inside it; the parts are processed side by side and the
        // separator's columns after them.  The tree is unique, so the result
        // does not depend on the schedule.
        std::vector<int32_t> parent(n, -1), anc(n, -1);
        auto liu = [&](int32_t c0, int32_t c1) {
            for (int32_t k = c0; k < c1; k++) {
                for (int64_t p = prp[k]; p < prp[k + 1]; p++) {
                    int32_t i = pci[p];
                    while (i != -1 && i < k) {
                        int32_t inext = anc[i];
                        anc[i] = k;
                        if (inext == -1) parent[i] = k;
                        i = inext;
                    }
                }
            }
        };
        {
            std::map<std::pair<int32_t, int32_t>, const NDState::Split *> split_of;
            for (const auto &sp : splits) split_of[{sp.lo, sp.m}] = &sp;
            // threads beyond the caller's, shared by every level of the
            // recursion: a split takes what it can use and gives it back
            std::atomic<int> spare{(int)spx::host_threads() - 1};
            auto take = [&](int want) {
                int have = spare.load();
                while (have > 0) {
                    const int got = std::min(have, want);
                    if (spare.compare_exchange_weak(have, have - got)) return got;
                }
                return 0;
            };
            std::function<void(int32_t, int32_t)> tree_range = [&](int32_t lo, int32_t m) {
                auto it = split_of.find({lo, m});
                if (it == split_of.end()) { liu(lo, lo + m); return; }
                const NDState::Split &sp = *it->second;
                const int np = (int)sp.parts.size();
                const int extra = np > 1 ? take(np - 1) : 0;
                std::atomic<int> nextp{0};
                auto work = [&] {
                    for (int q; (q = nextp.fetch_add(1)) < np;)
                        tree_range(sp.parts[q].first, sp.parts[q].second);
                };
                {
                    spx::TaskGroup g;
                    for (int t = 0; t < extra; t++) g.run(work);
                    work();
                    g.wait();
                }
                spare.fetch_add(extra);
                int32_t end = lo;
                for (const auto &pr : sp.parts) end = std::max(end, pr.first + pr.second);
                liu(end, lo + m);
            };
            tree_range(0, n);
        }

        // ---- 4. postorder, children in increasing order
        std::vector<int32_t> head(n, -1), next(n, -1), post(n), stack(n);
        for (int32_t j = n - 1; j >= 0; j--) {
            if (parent[j] == -1) continue;
            next[j] = head[parent[j]];
            head[parent[j]] = j;
        }
        {
            int32_t k = 0;
            for (int32_t r = 0; r < n; r++) {
                if (parent[r] != -1) continue;
                int32_t top = 0;
                stack[0] = r;
                while (top >= 0) {
                    int32_t p = stack[top];
                    int32_t c = head[p];
                    if (c == -1) {
                        top--;
                        post[k++] = p;
                    } else {
                        head[p] = next[c];
                        stack[++top] = c;
                    }
                }
            }
        }
        // relabel: final perm = perm0[post[.]]
        // (permutation scatters and gathers: every index is written once)
        std::vector<int32_t> ipost(n);
        S->perm = xalloc<int32_t>(n);
        S->iperm = xalloc<int32_t>(n);
        spx::parallel_ranges(n, kGrain, [&](int64_t lo, int64_t hi) {
            for (int64_t k = lo; k < hi; k++) {
                ipost[post[k]] = (int32_t)k;
                S->perm[k] = perm0[post[k]];
                S->iperm[perm0[post[k]]] = (int32_t)k;
            }
        });
        std::vector<int32_t> par(n);
        spx::parallel_ranges(n, kGrain, [&](int64_t lo, int64_t hi) {
            for (int64_t k = lo; k < hi; k++) {
                const int32_t p = parent[post[k]];
                par[k] = (p == -1) ? -1 : ipost[p];
            }
        });
        // adjacency in final numbering
        {
            std::vector<int64_t> rp2(n + 1, 0);
            for (int32_t k = 0; k < n; k++) rp2[k + 1] = rp2[k] + (prp[post[k] + 1] - prp[post[k]]);
            std::vector<int32_t> ci2(rp2[n]);
            spx::parallel_ranges(n, kGrain, [&](int64_t lo, int64_t hi) {
                for (int64_t k = lo; k < hi; k++) {
                    int64_t q = rp2[k];
                    for (int64_t p = prp[post[k]]; p < prp[post[k] + 1]; p++)
                        ci2[q++] = ipost[pci[p]];
                }
            });
            prp.swap(rp2);
            pci.swap(ci2);
        }

        // ---- 5. column counts (Gilbert, Ng and Peyton)
        // In postorder every tree of the elimination forest is a contiguous
        // range of columns ending at its root, and the algorithm reads and
        // writes only entries of the tree it is in: ranges of whole trees
        // are counted on separate threads.
        std::vector<int32_t> first(n, -1), maxfirst(n, -1), prevleaf(n, -1), ancestor(n);
        std::vector<int64_t> delta(n, 0), cc(n, 0);
        auto count_range = [&](int32_t c0, int32_t c1) {
            for (int32_t k = c0; k < c1; k++) {
                int32_t j = k;
                delta[j] = (first[j] == -1) ? 1 : 0;
                for (; j != -1 && first[j] == -1; j = par[j]) first[j] = k;
            }
            for (int32_t i = c0; i < c1; i++) ancestor[i] = i;
            for (int32_t j = c0; j < c1; j++) {
                if (par[j] != -1) delta[par[j]]--;
                for (int64_t p = prp[j]; p < prp[j + 1]; p++) {
                    int32_t i = pci[p];
                    int jleaf;
                    int32_t q = gnp_leaf(i, j, first.data(), maxfirst.data(), prevleaf.data(),
                                         ancestor.data(), &jleaf);
                    if (jleaf >= 1) delta[j]++;
                    if (jleaf == 2) delta[q]--;
                }
                if (par[j] != -1) ancestor[j] = par[j];
            }
            for (int32_t j = c0; j < c1; j++) cc[j] = delta[j];
            for (int32_t j = c0; j < c1; j++)
                if (par[j] != -1) cc[par[j]] += cc[j];
        };
        {
            // chunks of whole trees, about n / (4 threads) columns each
            const int32_t want = std::max<int32_t>(kGrain, n / (int32_t)(4 * spx::host_threads()));
            std::vector<std::pair<int32_t, int32_t>> chunks;
            int32_t c0 = 0;
            for (int32_t j = 0; j < n; j++)
                if (par[j] == -1 && (j + 1 - c0 >= want || j == n - 1)) {
                    chunks.push_back({c0, j + 1});
                    c0 = j + 1;
                }
            if (c0 < n) chunks.push_back({c0, n});
            std::atomic<size_t> nextc{0};
            auto worker = [&] {
                for (size_t q; (q = nextc.fetch_add(1)) < chunks.size();)
                    count_range(chunks[q].first, chunks[q].second);
            };
            const unsigned nth = (unsigned)std::min<size_t>(spx::host_threads(), chunks.size());
            spx::TaskGroup g(nth > 1);
            for (unsigned t = 1; t < nth; t++) g.run(worker);
            worker();
            g.wait();
        }

        // ---- 6. fundamental supernodes
        std::vector<int32_t> nchild(n, 0);
        for (int32_t j = 0; j < n; j++)
            if (par[j] != -1) nchild[par[j]]++;
        std::vector<int32_t> fs_first;
        fs_first.reserve(n / 2 + 1);
        for (int32_t j = 0; j < n; j++) {
            bool join = j > 0 && par[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1;
            if (!join) fs_first.push_back(j);
        }
        int32_t nfs = (int32_t)fs_first.size();
        fs_first.push_back(n);
        std::vector<int32_t> fs_of(n);
        for (int32_t s = 0; s < nfs; s++)
            for (int32_t j = fs_first[s]; j < fs_first[s + 1]; j++) fs_of[j] = s;
        std::vector<int32_t> fs_par(nfs);
        for (int32_t s = 0; s < nfs; s++) {
            int32_t last = fs_first[s + 1] - 1;
            fs_par[s] = (par[last] == -1) ? -1 : fs_of[par[last]];
        }

        // ---- 7. relaxed amalgamation (bottom-up; merge a child into its
        // parent when the child's columns immediately precede the parent's)
        std::vector<int32_t> mfirst(fs_first.begin(), fs_first.end() - 1);  // current first col
        std::vector<int32_t> mcols(nfs), mrows(nfs), rep(nfs);
        std::vector<double> mzeros(nfs, 0.0);
        for (int32_t s = 0; s < nfs; s++) {
            mcols[s] = fs_first[s + 1] - fs_first[s];
            mrows[s] = (int32_t)cc[fs_first[s]];
            rep[s] = s;
        }
        // rep[s]: the fundamental supernode that now heads s's merged group
        // (groups are merged upward; the parent's record stays the live one)
        std::vector<char> absorbed(nfs, 0);
        for (int32_t s = 0; s < nfs; s++) {
            int32_t p = fs_par[s];
            if (p < 0) continue;
            // live group of p is p itself (p has not been absorbed yet, since
            // p > s in postorder and merging only goes upward)
            int32_t cs = mcols[s], cp = mcols[p];
            if (mfirst[s] + cs != mfirst[p]) continue;  // not contiguous
            int32_t rs = mrows[s], rp = mrows[p];
            int32_t ns = cs + cp;
            int32_t rnew = cs + rp;
            double newz = (double)cs * (double)(cs + rp - rs);
            double totz = mzeros[s] + mzeros[p] + newz;
            double denom = (double)ns * (ns + 1) / 2.0 + (double)ns * (double)(rnew - ns);
            double z = denom > 0 ? totz / denom : 0.0;
            bool merge = (ns <= 4) || (ns <= 16 && z < 0.8) || (ns <= 48 && z < 0.1) ||
                         (z < 0.05);
            if (!merge) continue;
            mfirst[p] = mfirst[s];
            mcols[p] = ns;
            mrows[p] = rnew;
            mzeros[p] = totz;
            absorbed[s] = 1;
        }
        // final supernodes: the non-absorbed fundamental ones, in column order
        std::vector<int32_t> fin_of_fs(nfs, -1);
        std::vector<int32_t> sf;
        for (int32_t s = 0; s < nfs; s++) {
            if (absorbed[s]) continue;
            fin_of_fs[s] = (int32_t)sf.size();
            sf.push_back(mfirst[s]);
        }
        const int32_t ns = (int32_t)sf.size();
        // sort by first column (postorder guarantees increasing already, but be safe)
        std::vector<int32_t> order(ns);
        for (int32_t i = 0; i < ns; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return sf[a] < sf[b]; });
        std::vector<int32_t> rank(ns);
        for (int32_t i = 0; i < ns; i++) rank[order[i]] = i;
        S->nsuper = ns;
        S->sfirst = xalloc<int32_t>(ns + 1);
        for (int32_t i = 0; i < ns; i++) S->sfirst[i] = sf[order[i]];
        S->sfirst[ns] = n;
        S->col2sup = xalloc<int32_t>(n);
        for (int32_t s = 0; s < ns; s++)
            for (int32_t j = S->sfirst[s]; j < S->sfirst[s + 1]; j++) S->col2sup[j] = s;
        S->sparent = xalloc<int32_t>(ns);
        for (int32_t s = 0; s < ns; s++) {
            int32_t last = S->sfirst[s + 1] - 1;
            S->sparent[s] = (par[last] == -1) ? -1 : S->col2sup[par[last]];
        }

        // ---- 8. row structure of every supernode
        std::vector<int32_t> cptr(ns + 1, 0), clist(ns);
        for (int32_t s = 0; s < ns; s++)
            if (S->sparent[s] >= 0) cptr[S->sparent[s] + 1]++;
        for (int32_t s = 0; s < ns; s++) cptr[s + 1] += cptr[s];
        {
            std::vector<int32_t> fill(cptr.begin(), cptr.end() - 1);
            for (int32_t s = 0; s < ns; s++)
                if (S->sparent[s] >= 0) clist[fill[S->sparent[s]]++] = s;
        }
        // Rows of supernode s: its own columns, then every row >= its last
        // column that appears in A's pivot columns or in a child's rows,
        // ascending.  Supernodes are in postorder, so a subtree is a
        // contiguous range ending at its root; disjoint subtrees are built
        // on separate threads (each with its own mark array), then the
        // supernodes above them in order.  The lists are written in place
        // into S->rows at offsets from the row counts the amalgamation
        // predicts (a merged supernode's rows are its own columns and its
        // parent's rows, so the prediction is exact); should a list ever
        // come out at another length, every list is built again into
        // separate vectors and the offsets follow the lists.
        std::vector<int64_t> rptr(ns + 1, 0);
        for (int32_t s = 0; s < nfs; s++)
            if (!absorbed[s]) rptr[rank[fin_of_fs[s]] + 1] = mrows[s];
        for (int32_t s = 0; s < ns; s++) rptr[s + 1] += rptr[s];
        S->rows = xalloc<int32_t>(rptr[ns]);
        std::vector<std::vector<int32_t>> rs;          // only when a prediction fails
        bool flat = true;
        std::atomic<int> mismatch{0};
        auto build_rows = [&](int32_t s, std::vector<int32_t> &mark, std::vector<int32_t> &tmp) {
            int32_t f = S->sfirst[s], l = S->sfirst[s + 1];
            tmp.clear();
            for (int32_t j = f; j < l; j++) {
                for (int64_t p = prp[j]; p < prp[j + 1]; p++) {
                    int32_t i = pci[p];
                    if (i >= l && mark[i] != s) { mark[i] = s; tmp.push_back(i); }
                }
            }
            for (int32_t q = cptr[s]; q < cptr[s + 1]; q++) {
                int32_t c = clist[q];
                int32_t cc0 = S->sfirst[c + 1] - S->sfirst[c];
                const int32_t *rc = flat ? S->rows + rptr[c] : rs[c].data();
                const size_t nrc = flat ? (size_t)(rptr[c + 1] - rptr[c]) : rs[c].size();
                for (size_t p = (size_t)cc0; p < nrc; p++) {
                    int32_t i = rc[p];
                    if (i >= l && mark[i] != s) { mark[i] = s; tmp.push_back(i); }
                }
            }
            std::sort(tmp.begin(), tmp.end());
            const size_t len = (size_t)(l - f) + tmp.size();
            if (flat) {
                if ((int64_t)len != rptr[s + 1] - rptr[s]) { mismatch = 1; return; }
                int32_t *out = S->rows + rptr[s];
                for (int32_t j = f; j < l; j++) *out++ = j;
                std::copy(tmp.begin(), tmp.end(), out);
            } else {
                std::vector<int32_t> &out = rs[s];
                out.reserve(len);
                for (int32_t j = f; j < l; j++) out.push_back(j);
                out.insert(out.end(), tmp.begin(), tmp.end());
            }
        };
        {
            // subtree sizes and first descendants (postorder)
            std::vector<int32_t> fdesc(ns);
            for (int32_t s = 0; s < ns; s++) fdesc[s] = s;
            for (int32_t s = 0; s < ns; s++) {
                const int32_t p = S->sparent[s];
                if (p >= 0 && fdesc[s] < fdesc[p]) fdesc[p] = fdesc[s];
            }
            const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
            const int32_t target = std::max<int32_t>(256, ns / (int32_t)(4 * hw));
            std::vector<char> in_task(ns, 0);
            std::vector<int32_t> task_root;
            std::vector<int32_t> stack;
            for (int32_t s = 0; s < ns; s++)
                if (S->sparent[s] < 0) stack.push_back(s);
            while (!stack.empty()) {
                const int32_t s = stack.back();
                stack.pop_back();
                if (s - fdesc[s] + 1 <= target) {
                    task_root.push_back(s);
                    continue;
                }
                for (int32_t q = cptr[s]; q < cptr[s + 1]; q++) stack.push_back(clist[q]);
            }
            for (int32_t r : task_root)
                for (int32_t s = fdesc[r]; s <= r; s++) in_task[s] = 1;
            const unsigned nth = (hw > 1 && ns > 2048) ? hw : 1u;
            auto build_all = [&] {
                std::atomic<size_t> next{0};
                auto worker = [&] {
                    std::vector<int32_t> mark(n, -1), tmp;
                    for (size_t t; (t = next.fetch_add(1)) < task_root.size();) {
                        const int32_t r = task_root[t];
                        for (int32_t s = fdesc[r]; s <= r; s++) build_rows(s, mark, tmp);
                    }
                };
                std::vector<std::thread> th;
                for (unsigned i = 1; i < nth; i++) th.emplace_back(worker);
                worker();
                for (auto &t : th) t.join();
                std::vector<int32_t> mark(n, -1), tmp;
                for (int32_t s = 0; s < ns && !(flat && mismatch); s++)
                    if (!in_task[s]) build_rows(s, mark, tmp);
            };
            build_all();
            if (mismatch) {
                flat = false;
                rs.assign(ns, {});
                build_all();
                for (int32_t s = 0; s < ns; s++) rptr[s + 1] = rptr[s] + (int64_t)rs[s].size();
                free(S->rows);
                S->rows = nullptr;
                S->rows = xalloc<int32_t>(rptr[ns]);
                for (int32_t s = 0; s < ns; s++)
                    std::copy(rs[s].begin(), rs[s].end(), S->rows + rptr[s]);
                std::vector<std::vector<int32_t>>().swap(rs);
            }
        }
        const int64_t nrows_total = rptr[ns];
        S->rowptr = xalloc<int64_t>(ns + 1);
        memcpy(S->rowptr, rptr.data(), (ns + 1) * sizeof(int64_t));
        const int32_t *rows = S->rows;

        // ---- 9. relative maps into the parent's row list
        // (every child has one parent, so the parents' writes are disjoint)
        S->relmap = xalloc<int32_t>(nrows_total);
        std::fill(S->relmap, S->relmap + nrows_total, -1);
        spx::parallel_ranges(ns, kGrain, [&](int64_t lo, int64_t hi) {
            std::vector<int32_t> pos(n, -1);
            for (int64_t p = lo; p < hi; p++) {
                if (cptr[p] == cptr[p + 1]) continue;
                for (int64_t t = rptr[p]; t < rptr[p + 1]; t++) pos[rows[t]] = (int32_t)(t - rptr[p]);
                for (int32_t q = cptr[p]; q < cptr[p + 1]; q++) {
                    int32_t c = clist[q];
                    int32_t cc0 = S->sfirst[c + 1] - S->sfirst[c];
                    for (int64_t t = rptr[c] + cc0; t < rptr[c + 1]; t++) S->relmap[t] = pos[rows[t]];
                }
                for (int64_t t = rptr[p]; t < rptr[p + 1]; t++) pos[rows[t]] = -1;
            }
        });

        // ---- 10. levels, fronts, statistics
        std::vector<int32_t> lev(ns, 0);
        int32_t maxlev = 0;
        for (int32_t s = 0; s < ns; s++) {  // children precede parents
            int32_t p = S->sparent[s];
            if (p >= 0 && lev[p] < lev[s] + 1) lev[p] = lev[s] + 1;
            if (lev[s] > maxlev) maxlev = lev[s];
        }
        S->nlevels = maxlev + 1;
        S->level_ptr = xalloc<int32_t>(S->nlevels + 1);
        S->level_sup = xalloc<int32_t>(ns);
        for (int32_t l = 0; l <= S->nlevels; l++) S->level_ptr[l] = 0;
        for (int32_t s = 0; s < ns; s++) S->level_ptr[lev[s] + 1]++;
        for (int32_t l = 0; l < S->nlevels; l++) S->level_ptr[l + 1] += S->level_ptr[l];
        {
            std::vector<int32_t> fill(S->level_ptr, S->level_ptr + S->nlevels);
            for (int32_t s = 0; s < ns; s++) S->level_sup[fill[lev[s]]++] = s;
        }
        S->child_ptr = xalloc<int32_t>(ns + 1);
        S->child_list = xalloc<int32_t>(ns);
        memcpy(S->child_ptr, cptr.data(), (ns + 1) * sizeof(int32_t));
        memcpy(S->child_list, clist.data(), ns * sizeof(int32_t));
        S->frontptr = xalloc<int64_t>(ns + 1);
        S->frontptr[0] = 0;
        S->nnzL = 0;
        S->flops = 0;
        S->max_rows = 0;
        S->max_cols = 0;
        for (int32_t s = 0; s < ns; s++) {
            int64_t r = rptr[s + 1] - rptr[s];
            int64_t c = S->sfirst[s + 1] - S->sfirst[s];
            S->frontptr[s + 1] = S->frontptr[s] + r * r;
            S->nnzL += c * (c + 1) / 2 + (r - c) * c;
            double cd = (double)c, bd = (double)(r - c);
            S->flops += cd * cd * cd / 3.0 + bd * cd * cd + bd * (bd + 1) * cd;
            if (r > S->max_rows) S->max_rows = (int32_t)r;
            if (c > S->max_cols) S->max_cols = (int32_t)c;
        }
        S->front_total = S->frontptr[ns];
    } catch (const std::bad_alloc &) {
        spx_symbolic_free(S);
        return -2;
    }
    return 0;
}
