// Block shift-invert solve: X = (A + shift I)^{-1} B for NR right-hand sides
// (NR = 8, 16, 24 or 32) in one persistent launch.
//
// Included by multifrontal.cu inside its anonymous namespace: it runs the
// task queue of mf_solve_sf (same tasks, same per-supernode metadata, same
// dependency counters and chunk partial sums) with every vector entry of the
// single solve widened to a row of NR doubles: the intermediate yf, x and
// update vectors u are stored row-major with stride NR in factor order; the
// right-hand sides are read from, and the results written to, the caller's
// column-major arrays in the original order.  A task's
// product (rows x pivots) x (pivots x 1) becomes (rows x pivots) x
// (pivots x NR), so the panel G is read once for all NR columns and the
// level structure -- which bounds the single solve -- is paid once.
//
// Small supernodes (c <= 16, r <= 128) and tiny leaves run one per warp on
// the FP64 tensor cores (mma.sync m8n8k4): the forward product G (r x c) x
// F (c x NR) as 8-row tiles of G times 8-column chunks of F, the backward
// product G^T V as 4-row steps with the columns of V as the M side.  Each
// panel entry is loaded once per task, and the latency of a task does not
// grow with NR: a lane holds one row's 2 entries of every chunk.  Tiles of
// large supernodes run on the whole block with thread = (row or column
// group, right-hand side): every warp reads the same panel entries
// (shared-memory broadcasts) and distinct right-hand-side entries.

struct BSolveArgs {
    const SNode *meta;
    const STask *tasks;
    int ntasks, ns;
    const int32_t *bundle, *perm, *rows, *cptr, *cidx;
    const Real *G;
    double *u, *yf, *x;                  // rows of NR, factor order
    const int32_t *fc_base, *fc_n, *bc_base, *bc_n;
    double *fpart, *bpart;               // per strip slot: kST rows of NR
    int *fcnt, *bcnt;
    int *sync;                           // as SolveArgs::sync
    const STask *wtasks;                 // as SolveArgs::wtasks
    int nfw, nbw;
    // the caller's right-hand sides and results: nr columns, column-major,
    // original order (columns nr .. NR-1 read as zero and are not written);
    // every read of bc is in a forward task and every write of xc in a
    // backward task, which starts after the whole forward pass, so xc may
    // be bc
    const double *bc;
    double *xc;
    int64_t ldb, ldx;
    int nr;
    int accumulate;                      // xc += the solution (else xc = it)
    const int *skip;
};

// Column strides of the staged panel strip (forward: 128 columns of 64 rows;
// backward: 64 columns of 128 rows) and the row stride of the vector
// segment, padded so the fragment loads of a half warp (4 rows x 4 columns
// of 8-byte words, or 8 x 4 of 4-byte words) fall in distinct banks.  Each
// is a multiple of 16 bytes, as the bulk copies need.
constexpr int kGSF = sizeof(Real) == 8 ? kST + 4 : kST + 8;
constexpr int kGSB = sizeof(Real) == 8 ? kStrip + 4 : kStrip + 8;
template <int NR>
struct BShared {                         // one tile task of the block
    static constexpr int SEG = 16 * ((NR + 11) / 16) + 4;   // row stride of seg
    Real gbuf[kStrip * kGSF > kST * kGSB ? kStrip * kGSF : kST * kGSB];
    double seg[kStrip * SEG];            // f segment (forward) or v segment (backward)
};

template <int NR>
struct BWarpShared {                     // one warp task
    double f[kWarpMaxC][NR];             // forward: the pivot rows' f
    int idx[kWarpMaxR][kGW];             // forward: gather lists; backward: row indices
    int cnt[kWarpMaxR], e0[kWarpMaxR];
};

SPX_DEV double2 ldcg2(const double *p) { return __ldcg(reinterpret_cast<const double2 *>(p)); }
SPX_DEV void st2(double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); }
SPX_DEV double ldg_panel(const Real *p) { return (double)__ldg(p); }
// right-hand-side columns col, col + 1 of original row `row`
SPX_DEV double2 brhs2(const BSolveArgs &a, int64_t row, int col) {
    return make_double2(col < a.nr ? __ldg(a.bc + (int64_t)col * a.ldb + row) : 0.0,
                        col + 1 < a.nr ? __ldg(a.bc + (int64_t)(col + 1) * a.ldb + row) : 0.0);
}
// result column col of original row `row`
SPX_DEV void bout1(const BSolveArgs &a, int64_t row, int col, double v) {
    if (col < a.nr) {
        double *o = a.xc + (int64_t)col * a.ldx + row;
        *o = a.accumulate ? *o + v : v;
    }
}

SPX_DEV void bstage_list(const BSolveArgs &a, int64_t g, int *idx, int *n, int *e0) {
    const int b0 = a.cptr[g], b1 = a.cptr[g + 1];
    *n = b1 - b0;
    *e0 = b0;
    const int m = min(b1 - b0, kGW);
    for (int e = 0; e < m; e++) idx[e] = a.cidx[b0 + e];
}
SPX_DEV int blist_at(const BSolveArgs &a, const int *idx, int e0, int e) {
    return e < kGW ? idx[e] : a.cidx[e0 + e];
}

// ---- forward, one small supernode per warp:
//   f(0:c) = b(pivots) + the children's updates of the pivot rows (shared);
//   [x1; r2] = G f on the tensor cores, 8 rows of G per tile;
//   yf(pivots) = x1,  u = (children's updates of the rows below) - r2.
// Fragment layout of m8n8k4: lane = 4 gq + tq holds A[gq][tq], B[tq][gq]
// and D[gq][2 tq .. 2 tq + 1].
template <int NR>
SPX_DEV void bfwd_warp(const BSolveArgs &a, int s, BWarpShared<NR> &w) {
    constexpr int NCH = NR / 8, H = NR / 2;
    constexpr int PP = kWarpMaxC * H / 32;        // (pivot, column pair) items per lane
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
    // the pivots' right-hand-side rows and the gather lists do not depend
    // on the children: both are read before the wait
    double2 bv[PP];
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = lane + 32 * p, j = e / H, h = e % H;
        bv[p] = (j < c) ? brhs2(a, a.perm[first + j], 2 * h) : make_double2(0.0, 0.0);
    }
    if (nchild > 0)
        for (int i = lane; i < r; i += 32) bstage_list(a, g0 + i, w.idx[i], &w.cnt[i], &w.e0[i]);
    __syncwarp();
    if (nchild > 0) {
        if (lane == 0) wait_at_least(fcd + s, expect, err);
        __syncwarp();
    }
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = lane + 32 * p, j = e / H, h = e % H;
        if (j < c) {
            double2 v = bv[p];
            if (nchild > 0) {
                const int n = w.cnt[j], e0 = w.e0[j];
                for (int q = 0; q < n; q++) {
                    const double2 t = ldcg2(a.u + (int64_t)blist_at(a, w.idx[j], e0, q) * NR + 2 * h);
                    v.x += t.x;
                    v.y += t.y;
                }
            }
            w.f[j][2 * h] = v.x;
            w.f[j][2 * h + 1] = v.y;
        }
    }
    __syncwarp();
    const int nks = (c + 3) >> 2, nmt = (r + 7) >> 3;
    for (int mt = 0; mt < nmt; mt++) {
        const int i = mt * 8 + gq;                  // this lane's row of G and of the result
        double af[4];
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
            const int k = ks * 4 + tq;
            af[ks] = (ks < nks && k < c && i < r) ? ldg_panel(Gs + (int64_t)i + (int64_t)k * ldg)
                                                  : 0.0;
        }
        double2 add[NCH];
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) add[ch] = make_double2(0.0, 0.0);
        if (nchild > 0 && i >= c && i < r) {
            const int n = w.cnt[i], e0 = w.e0[i];
            for (int q = 0; q < n; q++) {
                const double *src = a.u + (int64_t)blist_at(a, w.idx[i], e0, q) * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++) {
                    const double2 t = ldcg2(src + 8 * ch);
                    add[ch].x += t.x;
                    add[ch].y += t.y;
                }
            }
        }
        double d[NCH][2];
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) d[ch][0] = d[ch][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
            if (ks < nks) {
                const int k = ks * 4 + tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++)
                    dmma(d[ch][0], d[ch][1], af[ks], k < c ? w.f[k][8 * ch + gq] : 0.0);
            }
        }
        if (i < r) {
            if (i < c) {
                double *dst = a.yf + (int64_t)(first + i) * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++) st2(dst + 8 * ch, d[ch][0], d[ch][1]);
            } else {
                double *dst = a.u + (m.uptr + (i - c)) * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++)
                    st2(dst + 8 * ch, add[ch].x - d[ch][0], add[ch].y - d[ch][1]);
            }
        }
    }
    __syncwarp();
    if (lane == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
}

// ---- backward, one small supernode per warp:  x1 = G^T v with
// v = [yf(pivots); -x(rows below)], on the tensor cores as D = v^T G:
// the M side is an 8-column chunk of v, N is 8 pivots, K runs over the rows
// four at a time.  The row indices are read before the wait.
template <int NR>
SPX_DEV void bbwd_warp(const BSolveArgs &a, int s, BWarpShared<NR> &w) {
    constexpr int NCH = NR / 8;
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
    int *ridx = &w.idx[0][0];
    for (int i = c + lane; i < r; i += 32) ridx[i] = rows[i];
    // the result's destinations: pivots 2 tq, 2 tq + 1 (+ 8)
    int pv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = (q >> 1) * 8 + 2 * tq + (q & 1);
        pv[q] = j < c ? a.perm[first + j] : 0;
    }
    __syncwarp();
    if (lane == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncwarp();
    const bool two = c > 8;
    const int nkk = (r + 3) >> 2;
    double d[NCH][2][2];
#pragma unroll
    for (int ch = 0; ch < NCH; ch++) d[ch][0][0] = d[ch][0][1] = d[ch][1][0] = d[ch][1][1] = 0.0;
#pragma unroll 2
    for (int ks = 0; ks < nkk; ks++) {
        const int i = ks * 4 + tq;
        double av[NCH];
        if (i < c) {
            const double *src = a.yf + (int64_t)(first + i) * NR + gq;
#pragma unroll
            for (int ch = 0; ch < NCH; ch++) av[ch] = __ldcg(src + 8 * ch);
        } else if (i < r) {
            const double *src = a.x + (int64_t)ridx[i] * NR + gq;
#pragma unroll
            for (int ch = 0; ch < NCH; ch++) av[ch] = -__ldcg(src + 8 * ch);
        } else {
#pragma unroll
            for (int ch = 0; ch < NCH; ch++) av[ch] = 0.0;
        }
        const double b0 = (i < r && gq < c) ? ldg_panel(Gs + (int64_t)i + (int64_t)gq * ldg) : 0.0;
        const double b1 = (two && i < r && 8 + gq < c)
                              ? ldg_panel(Gs + (int64_t)i + (int64_t)(8 + gq) * ldg) : 0.0;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) {
            dmma(d[ch][0][0], d[ch][0][1], av[ch], b0);
            if (two) dmma(d[ch][1][0], d[ch][1][1], av[ch], b1);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = (q >> 1) * 8 + 2 * tq + (q & 1);
        if (j >= c) continue;
        double *xr = a.x + (int64_t)(first + j) * NR + gq;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) {
            const double v = d[ch][q >> 1][q & 1];
            xr[8 * ch] = v;
            bout1(a, pv[q], 8 * ch + gq, v);
        }
    }
    __syncwarp();
    if (lane == 0) add_release(bdone + s, 1);
}

// ---- tiny leaves (r <= 24, c <= 6, no children): a bundle's leaves shared
// out over the block's warps, one leaf per warp at a time
template <int NR>
SPX_DEV void bfwd_leaves(const BSolveArgs &a, int boff, int bn, BWarpShared<NR> &w) {
    for (int li = threadIdx.x >> 5; li < bn; li += kSWarps) bfwd_warp<NR>(a, a.bundle[boff + li], w);
}

template <int NR>
SPX_DEV void bbwd_leaves(const BSolveArgs &a, int boff, int bn, BWarpShared<NR> &w) {
    for (int li = threadIdx.x >> 5; li < bn; li += kSWarps) bbwd_warp<NR>(a, a.bundle[boff + li], w);
}

// ---- tiny leaves eight to a warp: lanes 4 g .. 4 g + 3 take one leaf (live
// when the leaf exists), lane tq columns 2 tq, 2 tq + 1 of every 8-column
// chunk, with plain FP64 multiply-adds (a leaf's G is at most kTinyR x
// kTinyC).  Forward: [yf(pivots); -u] = G b(pivots) -- a leaf has no
// children to wait for.
template <int NR>
SPX_DEV void bfwd_leaf_group(const BSolveArgs &a, int s, bool live) {
    constexpr int NCH = NR / 8;
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns;
    const int tq = threadIdx.x & 3;
    int parent = -1;
    if (live) {
        const SNode m = a.meta[s];
        const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
        parent = m.b.x;
        const Real *Gs = a.G + m.p.x;
        int pr[kTinyC];
#pragma unroll
        for (int j = 0; j < kTinyC; j++) pr[j] = j < c ? a.perm[first + j] : 0;
#pragma unroll 1
        for (int ch = 0; ch < NCH; ch++) {
            const int col = 8 * ch + 2 * tq;
            double2 f[kTinyC];
#pragma unroll
            for (int j = 0; j < kTinyC; j++)
                f[j] = j < c ? brhs2(a, pr[j], col) : make_double2(0.0, 0.0);
#pragma unroll 2
            for (int i = 0; i < r; i++) {
                {
                    double x0 = 0.0, x1 = 0.0;
#pragma unroll
                    for (int j = 0; j < kTinyC; j++)
                        if (j < c) {
                            const double g = ldg_panel(Gs + (int64_t)i + (int64_t)j * ldg);
                            x0 += g * f[j].x;
                            x1 += g * f[j].y;
                        }
                    if (i < c) st2(a.yf + (int64_t)(first + i) * NR + col, x0, x1);
                    else st2(a.u + (m.uptr + (i - c)) * NR + col, -x0, -x1);
                }
            }
        }
    }
    __syncwarp();
    if (live && tq == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
}

// Backward: x(pivots) = G^T [yf(pivots); -x(rows below)] once the parent's
// backward has completed.
template <int NR>
SPX_DEV void bbwd_leaf_group(const BSolveArgs &a, int s, bool live) {
    constexpr int NCH = NR / 8;
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const int tq = threadIdx.x & 3;
    SNode m{};
    if (live) {
        m = a.meta[s];
        if (tq == 0) wait_at_least(m.b.x >= 0 ? bdone + m.b.x : fchk + s, m.bwd_expect, err);
    }
    __syncwarp();
    if (live) {
        const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
        const int32_t *rows = a.rows + m.p.y;
        const Real *Gs = a.G + m.p.x;
#pragma unroll 1
        for (int ch = 0; ch < NCH; ch++) {
            const int col = 8 * ch + 2 * tq;
            double2 acc[kTinyC];
#pragma unroll
            for (int j = 0; j < kTinyC; j++) acc[j] = make_double2(0.0, 0.0);
#pragma unroll 2
            for (int i = 0; i < r; i++) {
                {
                    double2 v;
                    if (i < c) {
                        v = ldcg2(a.yf + (int64_t)(first + i) * NR + col);
                    } else {
                        v = ldcg2(a.x + (int64_t)rows[i] * NR + col);
                        v.x = -v.x;
                        v.y = -v.y;
                    }
#pragma unroll
                    for (int j = 0; j < kTinyC; j++)
                        if (j < c) {
                            const double g = ldg_panel(Gs + (int64_t)i + (int64_t)j * ldg);
                            acc[j].x += g * v.x;
                            acc[j].y += g * v.y;
                        }
                }
            }
#pragma unroll
            for (int j = 0; j < kTinyC; j++)
                if (j < c) {
                    st2(a.x + (int64_t)(first + j) * NR + col, acc[j].x, acc[j].y);
                    const int pj = a.perm[first + j];
                    bout1(a, pj, col, acc[j].x);
                    bout1(a, pj, col + 1, acc[j].y);
                }
        }
    }
    __syncwarp();
    if (live && tq == 0) add_release(bdone + s, 1);
}


// ---- forward, rows [64 I, 64 I + 64) x a 128-column strip S of a large
// supernode's panel: (64 x 128) x (128 x NR) on the tensor cores, warp w
// holding rows 8 w .. 8 w + 7 of every 8-column chunk; the strip is staged
// into shared memory by bulk copies while the task waits for the children
template <int NR>
SPX_DEV void bfwd_tile(const BSolveArgs &a, int s, int I, int S, int chunk, BShared<NR> &sh,
                       unsigned long long *bar, uint32_t &phase, int *flag) {
    constexpr int NCH = NR / 8, H = NR / 2, SEG = BShared<NR>::SEG;
    constexpr int PP = kStrip * H / kSThreads;          // (column, pair) items per thread
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const int i0 = I * kST, j0 = S * kStrip;
    const int jn = min(kStrip, c - j0);
    const int hcopy = min(kST, ldg - i0);
    stage_panel(sh.gbuf, kGSF, a.G + m.p.x, ldg, i0, hcopy, j0, jn, bar);
    const int t = threadIdx.x;
    // the strip's right-hand-side rows, read before the wait
    double2 bv[PP];
    // and the children's gather lists of those rows -- their bounds and first
    // two entries -- so that after the wait only the update rows are read
    int qb[PP], qe[PP], q0i[PP], q1i[PP];
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = t + kSThreads * p, jj = e / H, h = e % H;
        bv[p] = (jj < jn) ? brhs2(a, a.perm[first + j0 + jj], 2 * h) : make_double2(0.0, 0.0);
        qb[p] = qe[p] = q0i[p] = q1i[p] = 0;
        if (jj < jn && nchild > 0) {
            const int64_t g = g0 + j0 + jj;
            qb[p] = a.cptr[g];
            qe[p] = a.cptr[g + 1];
            if (qb[p] < qe[p]) q0i[p] = a.cidx[qb[p]];
            if (qb[p] + 1 < qe[p]) q1i[p] = a.cidx[qb[p] + 1];
        }
    }
    // the same for this lane's row of the update part, which the block that
    // completes the row chunk gathers
    int ub = 0, ue = 0, u0i = 0, u1i = 0;
    {
        const int ur = i0 + (t >> 5) * 8 + ((t & 31) >> 2);
        if (nchild > 0 && ur >= c && ur < r) {
            const int64_t g = g0 + ur;
            ub = a.cptr[g];
            ue = a.cptr[g + 1];
            if (ub < ue) u0i = a.cidx[ub];
            if (ub + 1 < ue) u1i = a.cidx[ub + 1];
        }
    }
    if (nchild > 0 && t == 0) wait_at_least(fcd + s, expect, err);
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = t + kSThreads * p, jj = e / H, h = e % H;
        double2 v = bv[p];
        if (jj < jn && nchild > 0) {
            for (int q = qb[p]; q < qe[p]; q++) {
                const int ci = q == qb[p] ? q0i[p] : (q == qb[p] + 1 ? q1i[p] : a.cidx[q]);
                const double2 u = ldcg2(a.u + (int64_t)ci * NR + 2 * h);
                v.x += u.x;
                v.y += u.y;
            }
        }
        sh.seg[jj * SEG + 2 * h] = v.x;
        sh.seg[jj * SEG + 2 * h + 1] = v.y;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    const int lane = t & 31, wid = t >> 5, gq = lane >> 2, tq = lane & 3;
    const int row = wid * 8 + gq;                        // this lane's row in the chunk
    double d[NCH][2];
#pragma unroll
    for (int ch = 0; ch < NCH; ch++) d[ch][0] = d[ch][1] = 0.0;
    const int nks = (jn + 3) >> 2;
#pragma unroll 4
    for (int ks = 0; ks < nks; ks++) {
        const int k = ks * 4 + tq;
        const double av = k < jn ? (double)sh.gbuf[k * kGSF + row] : 0.0;
        const double *sb = sh.seg + (ks * 4 + tq) * SEG + gq;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) dmma(d[ch][0], d[ch][1], av, sb[8 * ch]);
    }
    const int nt = a.fc_n[chunk];
    if (nt > 1) {
        double *slot = a.fpart + (int64_t)(a.fc_base[chunk] + S) * kST * NR + row * NR + 2 * tq;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) st2(slot + 8 * ch, d[ch][0], d[ch][1]);
    }
    // a row chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.fcnt + chunk, nt, flag)) {
        const int ii = i0 + row;
        if (ii < r) {
            if (nt > 1) {
                const double *p0 = a.fpart + (int64_t)a.fc_base[chunk] * kST * NR + row * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++) d[ch][0] = d[ch][1] = 0.0;
                for (int q = 0; q < nt; q++)
#pragma unroll
                    for (int ch = 0; ch < NCH; ch++) {
                        const double2 v = ldcg2(p0 + (int64_t)q * kST * NR + 8 * ch);
                        d[ch][0] += v.x;
                        d[ch][1] += v.y;
                    }
            }
            if (ii < c) {
                double *dst = a.yf + (int64_t)(first + ii) * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++) st2(dst + 8 * ch, d[ch][0], d[ch][1]);
            } else {
                double2 add[NCH];
#pragma unroll
                for (int ch = 0; ch < NCH; ch++) add[ch] = make_double2(0.0, 0.0);
                if (nchild > 0) {
                    for (int q = ub; q < ue; q++) {
                        const int ci = q == ub ? u0i : (q == ub + 1 ? u1i : a.cidx[q]);
                        const double *src = a.u + (int64_t)ci * NR + 2 * tq;
#pragma unroll
                        for (int ch = 0; ch < NCH; ch++) {
                            const double2 u = ldcg2(src + 8 * ch);
                            add[ch].x += u.x;
                            add[ch].y += u.y;
                        }
                    }
                }
                double *dst = a.u + (m.uptr + (ii - c)) * NR + 2 * tq;
#pragma unroll
                for (int ch = 0; ch < NCH; ch++)
                    st2(dst + 8 * ch, add[ch].x - d[ch][0], add[ch].y - d[ch][1]);
            }
        }
        __syncthreads();
        // one completed row chunk: the parent counts every chunk of every child
        if (t == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
    }
    __syncthreads();
}

// ---- backward, columns [64 J, 64 J + 64) x a 128-row strip S of a large
// supernode's panel: D = v^T G_strip on the tensor cores (M: 8-column
// chunks of v, N: warp w's 8 pivots 8 w .. 8 w + 7, K: the strip's rows)
template <int NR>
SPX_DEV void bbwd_tile(const BSolveArgs &a, int s, int J, int S, int chunk, BShared<NR> &sh,
                       unsigned long long *bar, uint32_t &phase, int *flag) {
    constexpr int NCH = NR / 8, H = NR / 2, SEG = BShared<NR>::SEG;
    constexpr int PP = kStrip * H / kSThreads;
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const int i0 = S * kStrip, j0 = J * kST;
    const int in = min(kStrip, r - i0), jn = min(kST, c - j0);
    const int hcopy = min(kStrip, ldg - i0);
    stage_panel(sh.gbuf, kGSB, a.G + m.p.x, ldg, i0, hcopy, j0, jn, bar);
    const int t = threadIdx.x;
    // row indices of the strip's rows below the pivots, read before the wait
    int ri[PP];
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = t + kSThreads * p, ii = e / H, gi = i0 + ii;
        ri[p] = (ii < in && gi >= c) ? rows[gi] : 0;
    }
    if (t == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PP; p++) {
        const int e = t + kSThreads * p, ii = e / H, h = e % H, gi = i0 + ii;
        double2 v = make_double2(0.0, 0.0);
        if (ii < in) {
            if (gi < c) {
                v = ldcg2(a.yf + (int64_t)(first + gi) * NR + 2 * h);
            } else {
                v = ldcg2(a.x + (int64_t)ri[p] * NR + 2 * h);
                v.x = -v.x;
                v.y = -v.y;
            }
        }
        sh.seg[ii * SEG + 2 * h] = v.x;
        sh.seg[ii * SEG + 2 * h + 1] = v.y;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    const int lane = t & 31, wid = t >> 5, gq = lane >> 2, tq = lane & 3;
    const int pc = wid * 8 + gq;                         // this lane's pivot column (B side)
    double d[NCH][2];
#pragma unroll
    for (int ch = 0; ch < NCH; ch++) d[ch][0] = d[ch][1] = 0.0;
    const int nks = (in + 3) >> 2;
#pragma unroll 4
    for (int ks = 0; ks < nks; ks++) {
        const int k = ks * 4 + tq;
        const double bg = (k < in && pc < jn) ? (double)sh.gbuf[pc * kGSB + k] : 0.0;
        const double *sa = sh.seg + k * SEG + gq;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) dmma(d[ch][0], d[ch][1], sa[8 * ch], bg);
    }
    // lane holds D[col = 8 ch + gq][pivot = 8 wid + 2 tq + e]
    const int nt = a.bc_n[chunk];
    if (nt > 1) {
        double *slot = a.bpart + (int64_t)(a.bc_base[chunk] + (S - (j0 / kStrip))) * kST * NR;
#pragma unroll
        for (int e = 0; e < 2; e++)
#pragma unroll
            for (int ch = 0; ch < NCH; ch++)
                slot[(wid * 8 + 2 * tq + e) * NR + 8 * ch + gq] = d[ch][e];
    }
    // a column chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.bcnt + chunk, nt, flag)) {
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int jj = wid * 8 + 2 * tq + e;
            if (jj >= jn) continue;
            const int64_t orow = a.perm[first + j0 + jj];
#pragma unroll
            for (int ch = 0; ch < NCH; ch++) {
                double rr = d[ch][e];
                if (nt > 1) {
                    const double *p0 = a.bpart + (int64_t)a.bc_base[chunk] * kST * NR + jj * NR +
                                       8 * ch + gq;
                    rr = 0.0;
                    for (int q = 0; q < nt; q++) rr += __ldcg(p0 + (int64_t)q * kST * NR);
                }
                a.x[(int64_t)(first + j0 + jj) * NR + 8 * ch + gq] = rr;
                bout1(a, orow, 8 * ch + gq, rr);
            }
        }
        __syncthreads();
        // one completed column chunk: the children count every chunk
        if (t == 0) add_release(bdone + s, 1);
    }
    __syncthreads();
}

// Warp tasks of one phase (as solve_warp_tasks): a small supernode, or up to
// 32 tiny leaves solved one after another by the warp.
template <int NR>
SPX_DEV void bsolve_warp_tasks(const BSolveArgs &a, const STask *tq, int nt, int *ctr,
                               BWarpShared<NR> &w) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(ctr, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nt) break;
        const STask tk = tq[t];
        const bool fwd = tk.a.x == ST_FWD_BUNDLE || tk.a.x == ST_FWD_THREADS;
        if (tk.a.x == ST_FWD_THREADS || tk.a.x == ST_BWD_THREADS) {
            // tiny leaves: eight at a time, four lanes each
            const int g = lane >> 2;
            for (int p = 0; p < tk.b.z; p += 8) {
                const bool live = p + g < tk.b.z;
                const int s = live ? a.bundle[tk.b.y + p + g] : 0;
                if (fwd) bfwd_leaf_group<NR>(a, s, live);
                else bbwd_leaf_group<NR>(a, s, live);
            }
        } else {
            for (int q = 0; q < tk.b.z; q++) {
                if (fwd) bfwd_warp<NR>(a, a.bundle[tk.b.y + q], w);
                else bbwd_warp<NR>(a, a.bundle[tk.b.y + q], w);
            }
        }
        __syncwarp();
    }
}

template <int NR>
__global__ void __launch_bounds__(kSThreads, 2) mf_bsolve(BSolveArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int s_task, s_flag;
    __shared__ __align__(8) unsigned long long s_bar;
    BShared<NR> &sh = *reinterpret_cast<BShared<NR> *>(smem_raw);
    if (a.skip && *(volatile const int *)a.skip) return;
    const int wid = threadIdx.x >> 5;
    BWarpShared<NR> &ws = reinterpret_cast<BWarpShared<NR> *>(smem_raw)[wid];
    uint32_t phase = 0;
    if (threadIdx.x == 0) mbar_init(&s_bar);
    bsolve_warp_tasks<NR>(a, a.wtasks, a.nfw, a.sync + 1 + a.ns, ws);
    __syncthreads();
    fence_proxy_async();
    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(a.sync, 1);
        __syncthreads();
        const int t = s_task;
        __syncthreads();
        if (t >= a.ntasks) break;
        const STask tk = a.tasks[t];
        switch (tk.a.x) {
            case ST_FWD_BUNDLE:
                if (wid < tk.b.z) bfwd_warp<NR>(a, a.bundle[tk.b.y + wid], ws);
                break;
            case ST_FWD_TILE:
                bfwd_tile<NR>(a, tk.a.y, tk.a.z, tk.a.w, tk.b.x, sh, &s_bar, phase, &s_flag);
                break;
            case ST_BWD_BUNDLE:
                if (wid < tk.b.z) bbwd_warp<NR>(a, a.bundle[tk.b.y + wid], ws);
                break;
            case ST_FWD_THREADS:
                bfwd_leaves<NR>(a, tk.b.y, tk.b.z, ws);
                break;
            case ST_BWD_THREADS:
                bbwd_leaves<NR>(a, tk.b.y, tk.b.z, ws);
                break;
            default:
                bbwd_tile<NR>(a, tk.a.y, tk.a.z, tk.a.w, tk.b.x, sh, &s_bar, phase, &s_flag);
                break;
        }
        __syncthreads();
        // shared memory read by this task may be refilled by the async
        // proxy in the next one
        fence_proxy_async();
    }
    bsolve_warp_tasks<NR>(a, a.wtasks + a.nfw, a.nbw, a.sync + 1 + 4 * a.ns, ws);
}

template <int NR>
constexpr size_t bsolve_smem_bytes() {
    return sizeof(BShared<NR>) > sizeof(BWarpShared<NR>) * kSWarps
               ? sizeof(BShared<NR>) : sizeof(BWarpShared<NR>) * kSWarps;
}
