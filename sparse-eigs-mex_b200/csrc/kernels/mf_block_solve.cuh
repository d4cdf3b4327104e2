// Block shift-invert solve: X = (A + shift I)^{-1} B for NR right-hand sides
// (NR = 8, 16 or 32) in one persistent launch.
//
// Included by multifrontal.cu inside its anonymous namespace: it runs the
// task queue of mf_solve_sf (same tasks, same per-supernode metadata, same
// dependency counters and chunk partial sums) with every vector entry of the
// single solve widened to a row of NR doubles, stored row-major with stride
// NR: the right-hand sides and the result in the original order, the
// intermediate yf, x and update vectors u in factor order.  A task's
// product (rows x pivots) x (pivots x 1) becomes (rows x pivots) x
// (pivots x NR), so the panel G is read once for all NR columns and the
// level structure -- which bounds the single solve -- is paid once.
//
// Thread mapping.  Small supernodes (c <= 16, r <= 128) and tiny leaves run
// one per warp with lane = (row group, column): NR lanes per row group,
// 32 / NR row groups per warp.  Tiles of large supernodes run on the whole
// block with thread = (row or column group, right-hand side): every warp
// reads the same panel entries (shared-memory broadcasts) and distinct
// right-hand-side entries (consecutive, conflict-free).

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
    const double *b;                     // n rows of NR, original order
    double *out;                         // n rows of NR, original order
    const int *skip;
};

template <int NR>
struct BShared {                         // one tile task of the block
    Real gbuf[kStrip * kST];             // staged panel strip, as in SolveShared
    double seg[kStrip][NR];              // f segment (forward) or v segment (backward)
};

// sum of the children's update rows listed for front row g, column col
template <int NR>
SPX_DEV double bsum_list(const BSolveArgs &a, int64_t g, int col) {
    double acc = 0.0;
    const int e1 = a.cptr[g + 1];
    for (int e = a.cptr[g]; e < e1; e++) acc += __ldcg(a.u + (int64_t)a.cidx[e] * NR + col);
    return acc;
}

// ---- forward, one small supernode per warp
template <int NR>
SPX_DEV void bfwd_warp(const BSolveArgs &a, int s, double (*fw)[NR]) {
    constexpr int GW = 32 / NR;
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31, col = lane % NR, grp = lane / NR;
    if (nchild > 0) {
        if (lane == 0) wait_at_least(fcd + s, expect, err);
        __syncwarp();
    }
    // f(0:c) = b(pivots) + the children's updates of the pivot rows
    for (int j = grp; j < c; j += GW) {
        double v = a.b[(int64_t)a.perm[first + j] * NR + col];
        if (nchild > 0) v += bsum_list<NR>(a, g0 + j, col);
        fw[j][col] = v;
    }
    __syncwarp();
    for (int i = grp; i < r; i += GW) {
        // the row's panel entries are loaded together before they are used
        double g[kWarpMaxC];
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++)
            g[j] = (j < c) ? (double)Gs[(int64_t)i + (int64_t)j * ldg] : 0.0;
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++)
            if (j < c) acc += g[j] * fw[j][col];
        if (i < c) {
            a.yf[(int64_t)(first + i) * NR + col] = acc;
        } else {
            const double add = nchild > 0 ? bsum_list<NR>(a, g0 + i, col) : 0.0;
            a.u[(m.uptr + (i - c)) * NR + col] = add - acc;
        }
    }
    __syncwarp();
    if (lane == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
}

// ---- backward, one small supernode per warp
template <int NR>
SPX_DEV void bbwd_warp(const BSolveArgs &a, int s) {
    constexpr int GW = 32 / NR;
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31, col = lane % NR, grp = lane / NR;
    if (lane == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncwarp();
    double p[kWarpMaxC];
#pragma unroll
    for (int j = 0; j < kWarpMaxC; j++) p[j] = 0.0;
    for (int i = grp; i < r; i += GW) {
        const double v = (i < c) ? __ldcg(a.yf + (int64_t)(first + i) * NR + col)
                                 : -__ldcg(a.x + (int64_t)rows[i] * NR + col);
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++)
            if (j < c) p[j] += (double)Gs[(int64_t)i + (int64_t)j * ldg] * v;
    }
    // add the row groups' partial sums (lanes col, col + NR, ...)
#pragma unroll
    for (int off = NR; off < 32; off <<= 1)
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++) p[j] += __shfl_xor_sync(0xffffffffu, p[j], off);
    if (grp == 0) {
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++)
            if (j < c) {
                a.x[(int64_t)(first + j) * NR + col] = p[j];
                a.out[(int64_t)a.perm[first + j] * NR + col] = p[j];
            }
    }
    __syncwarp();
    if (lane == 0) add_release(bdone + s, 1);
}

// ---- tiny leaves (r <= 24, c <= 6, no children): 32 / NR leaves per warp
// at a time, the bundle's leaves shared out over the block's warps
template <int NR>
SPX_DEV void bfwd_leaves(const BSolveArgs &a, int boff, int bn) {
    constexpr int GW = 32 / NR;
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns;
    const int lane = threadIdx.x & 31, col = lane % NR, grp = lane / NR, wid = threadIdx.x >> 5;
    const int per_pass = kSWarps * GW;
    for (int base = 0; base < bn; base += per_pass) {
        const int li = base + wid * GW + grp;
        const bool on = li < bn;
        int s = 0, parent = -1;
        if (on) {
            s = a.bundle[boff + li];
            const SNode m = a.meta[s];
            const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
            parent = m.b.x;
            const Real *Gs = a.G + m.p.x;
            double f[kTinyC];
#pragma unroll
            for (int j = 0; j < kTinyC; j++)
                f[j] = (j < c) ? a.b[(int64_t)a.perm[first + j] * NR + col] : 0.0;
            for (int i = 0; i < r; i++) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < kTinyC; j++)
                    if (j < c) acc += (double)Gs[(int64_t)i + (int64_t)j * ldg] * f[j];
                if (i < c) a.yf[(int64_t)(first + i) * NR + col] = acc;
                else a.u[(m.uptr + (i - c)) * NR + col] = -acc;
            }
        }
        __syncwarp();
        if (on && col == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
    }
}

template <int NR>
SPX_DEV void bbwd_leaves(const BSolveArgs &a, int boff, int bn) {
    constexpr int GW = 32 / NR;
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const int lane = threadIdx.x & 31, col = lane % NR, grp = lane / NR, wid = threadIdx.x >> 5;
    const int per_pass = kSWarps * GW;
    for (int base = 0; base < bn; base += per_pass) {
        const int li = base + wid * GW + grp;
        const bool on = li < bn;
        int s = 0;
        SNode m;
        if (on) {
            s = a.bundle[boff + li];
            m = a.meta[s];
            if (col == 0)
                wait_at_least(m.b.x >= 0 ? bdone + m.b.x : fchk + s, m.bwd_expect, err);
        }
        __syncwarp();
        if (on) {
            const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
            const int32_t *rows = a.rows + m.p.y;
            const Real *Gs = a.G + m.p.x;
            double p[kTinyC];
#pragma unroll
            for (int j = 0; j < kTinyC; j++) p[j] = 0.0;
            for (int i = 0; i < r; i++) {
                const double v = (i < c) ? __ldcg(a.yf + (int64_t)(first + i) * NR + col)
                                         : -__ldcg(a.x + (int64_t)rows[i] * NR + col);
#pragma unroll
                for (int j = 0; j < kTinyC; j++)
                    if (j < c) p[j] += (double)Gs[(int64_t)i + (int64_t)j * ldg] * v;
            }
#pragma unroll
            for (int j = 0; j < kTinyC; j++)
                if (j < c) {
                    a.x[(int64_t)(first + j) * NR + col] = p[j];
                    a.out[(int64_t)a.perm[first + j] * NR + col] = p[j];
                }
        }
        __syncwarp();
        if (on && col == 0) add_release(bdone + s, 1);
    }
}

// ---- forward, rows [64 I, 64 I + 64) x a 128-column strip S of a large
// supernode's panel: (64 x 128) x (128 x NR), the strip staged into shared
// memory by bulk copies while the task waits for the children
template <int NR>
SPX_DEV void bfwd_tile(const BSolveArgs &a, int s, int I, int S, int chunk, BShared<NR> &sh,
                       unsigned long long *bar, uint32_t &phase, int *flag) {
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const int i0 = I * kST, j0 = S * kStrip;
    const int jn = min(kStrip, c - j0);
    const int hcopy = min(kST, ldg - i0);
    stage_panel(sh.gbuf, kST, a.G + m.p.x, ldg, i0, hcopy, j0, jn, bar);
    const int t = threadIdx.x;
    if (nchild > 0 && t == 0) wait_at_least(fcd + s, expect, err);
    __syncthreads();
    for (int e = t; e < kStrip * NR; e += kSThreads) {
        const int jj = e / NR, col = e % NR;
        double v = 0.0;
        if (jj < jn) {
            v = a.b[(int64_t)a.perm[first + j0 + jj] * NR + col];
            if (nchild > 0) v += bsum_list<NR>(a, g0 + j0 + jj, col);
        }
        sh.seg[jj][col] = v;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    constexpr int RPT = kST * NR / kSThreads;   // rows per thread
    const int col = t % NR, rg = t / NR;
    double acc[RPT];
#pragma unroll
    for (int k = 0; k < RPT; k++) acc[k] = 0.0;
    for (int jj = 0; jj < jn; jj++) {
        const double f = sh.seg[jj][col];
        const Real *gc = sh.gbuf + jj * kST + rg * RPT;
#pragma unroll
        for (int k = 0; k < RPT; k++) acc[k] += (double)gc[k] * f;
    }
    const int nt = a.fc_n[chunk];
    if (nt > 1) {
        double *slot = a.fpart + (int64_t)(a.fc_base[chunk] + S) * kST * NR;
#pragma unroll
        for (int k = 0; k < RPT; k++) slot[(rg * RPT + k) * NR + col] = acc[k];
    }
    // a row chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.fcnt + chunk, nt, flag)) {
#pragma unroll
        for (int k = 0; k < RPT; k++) {
            const int ii = i0 + rg * RPT + k;
            if (ii >= r) continue;
            double rr = acc[k];
            if (nt > 1) {
                const double *p0 = a.fpart + (int64_t)a.fc_base[chunk] * kST * NR +
                                   (rg * RPT + k) * NR + col;
                rr = 0.0;
                for (int q = 0; q < nt; q++) rr += __ldcg(p0 + (int64_t)q * kST * NR);
            }
            if (ii < c) {
                a.yf[(int64_t)(first + ii) * NR + col] = rr;
            } else {
                const double add = nchild > 0 ? bsum_list<NR>(a, g0 + ii, col) : 0.0;
                a.u[(m.uptr + (ii - c)) * NR + col] = add - rr;
            }
        }
        __syncthreads();
        // one completed row chunk: the parent counts every chunk of every child
        if (t == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
    }
    __syncthreads();
}

// ---- backward, columns [64 J, 64 J + 64) x a 128-row strip S of a large
// supernode's panel: (64 x 128) x (128 x NR) with the strip transposed
template <int NR>
SPX_DEV void bbwd_tile(const BSolveArgs &a, int s, int J, int S, int chunk, BShared<NR> &sh,
                       unsigned long long *bar, uint32_t &phase, int *flag) {
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const int i0 = S * kStrip, j0 = J * kST;
    const int in = min(kStrip, r - i0), jn = min(kST, c - j0);
    const int hcopy = min(kStrip, ldg - i0);
    stage_panel(sh.gbuf, kStrip, a.G + m.p.x, ldg, i0, hcopy, j0, jn, bar);
    const int t = threadIdx.x;
    if (t == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncthreads();
    for (int e = t; e < kStrip * NR; e += kSThreads) {
        const int ii = e / NR, col = e % NR, gi = i0 + ii;
        double v = 0.0;
        if (ii < in)
            v = (gi < c) ? __ldcg(a.yf + (int64_t)(first + gi) * NR + col)
                         : -__ldcg(a.x + (int64_t)rows[gi] * NR + col);
        sh.seg[ii][col] = v;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    constexpr int CPT = kST * NR / kSThreads;   // columns per thread
    const int col = t % NR, cg = t / NR;
    double acc[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) acc[k] = 0.0;
    for (int ii = 0; ii < in; ii++) {
        const double v = sh.seg[ii][col];
#pragma unroll
        for (int k = 0; k < CPT; k++) acc[k] += (double)sh.gbuf[(cg * CPT + k) * kStrip + ii] * v;
    }
    const int nt = a.bc_n[chunk];
    if (nt > 1) {
        double *slot = a.bpart + (int64_t)(a.bc_base[chunk] + (S - (j0 / kStrip))) * kST * NR;
#pragma unroll
        for (int k = 0; k < CPT; k++) slot[(cg * CPT + k) * NR + col] = acc[k];
    }
    // a column chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.bcnt + chunk, nt, flag)) {
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            const int jj = cg * CPT + k;
            if (jj >= jn) continue;
            double rr = acc[k];
            if (nt > 1) {
                const double *p0 = a.bpart + (int64_t)a.bc_base[chunk] * kST * NR + jj * NR + col;
                rr = 0.0;
                for (int q = 0; q < nt; q++) rr += __ldcg(p0 + (int64_t)q * kST * NR);
            }
            a.x[(int64_t)(first + j0 + jj) * NR + col] = rr;
            a.out[(int64_t)a.perm[first + j0 + jj] * NR + col] = rr;
        }
        __syncthreads();
        // one completed column chunk: the children count every chunk
        if (t == 0) add_release(bdone + s, 1);
    }
    __syncthreads();
}

template <int NR>
__global__ void __launch_bounds__(kSThreads, 2) mf_bsolve(BSolveArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int s_task, s_flag;
    __shared__ __align__(8) unsigned long long s_bar;
    BShared<NR> &sh = *reinterpret_cast<BShared<NR> *>(smem_raw);
    if (a.skip && *(volatile const int *)a.skip) return;
    const int wid = threadIdx.x >> 5;
    double(*fw)[NR] = reinterpret_cast<double(*)[NR]>(smem_raw) + wid * kWarpMaxC;
    uint32_t phase = 0;
    if (threadIdx.x == 0) mbar_init(&s_bar);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(a.sync, 1);
        __syncthreads();
        const int t = s_task;
        __syncthreads();
        if (t >= a.ntasks) break;
        const STask tk = a.tasks[t];
        switch (tk.a.x) {
            case ST_FWD_BUNDLE:
                if (wid < tk.b.z) bfwd_warp<NR>(a, a.bundle[tk.b.y + wid], fw);
                break;
            case ST_FWD_TILE:
                bfwd_tile<NR>(a, tk.a.y, tk.a.z, tk.a.w, tk.b.x, sh, &s_bar, phase, &s_flag);
                break;
            case ST_BWD_BUNDLE:
                if (wid < tk.b.z) bbwd_warp<NR>(a, a.bundle[tk.b.y + wid]);
                break;
            case ST_FWD_THREADS:
                bfwd_leaves<NR>(a, tk.b.y, tk.b.z);
                break;
            case ST_BWD_THREADS:
                bbwd_leaves<NR>(a, tk.b.y, tk.b.z);
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
}

template <int NR>
constexpr size_t bsolve_smem_bytes() {
    return sizeof(BShared<NR>) > sizeof(double) * kWarpMaxC * NR * kSWarps
               ? sizeof(BShared<NR>) : sizeof(double) * kWarpMaxC * NR * kSWarps;
}

// Column-major n x nr (leading dimension ld) <-> row-major n x NR (stride
// NR, columns nr..NR-1 zero on the way in).  A block of 256 threads moves 32
// rows through shared memory so both sides are read and written in
// contiguous runs.
template <int NR>
__global__ void __launch_bounds__(256) bs_to_rows(int n, int nr, const double *B, int64_t ld,
                                                  double *R, const int *skip) {
    __shared__ double tile[32][NR + 1];
    if (skip && *(volatile const int *)skip) return;
    const int r0 = blockIdx.x * 32;
    for (int e = threadIdx.x; e < 32 * NR; e += blockDim.x) {
        const int i = e % 32, c = e / 32;     // consecutive threads: consecutive rows
        tile[i][c] = (r0 + i < n && c < nr) ? B[(int64_t)(r0 + i) + (int64_t)c * ld] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * NR; e += blockDim.x) {
        const int i = e / NR, c = e % NR;     // consecutive threads: one row's columns
        if (r0 + i < n) R[(int64_t)(r0 + i) * NR + c] = tile[i][c];
    }
}

template <int NR>
__global__ void __launch_bounds__(256) bs_from_rows(int n, int nr, const double *R, double *X,
                                                    int64_t ld, const int *skip) {
    __shared__ double tile[32][NR + 1];
    if (skip && *(volatile const int *)skip) return;
    const int r0 = blockIdx.x * 32;
    for (int e = threadIdx.x; e < 32 * NR; e += blockDim.x) {
        const int i = e / NR, c = e % NR;
        tile[i][c] = (r0 + i < n) ? R[(int64_t)(r0 + i) * NR + c] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * NR; e += blockDim.x) {
        const int i = e % 32, c = e / 32;
        if (r0 + i < n && c < nr) X[(int64_t)(r0 + i) + (int64_t)c * ld] = tile[i][c];
    }
}
