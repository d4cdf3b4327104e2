// Device multifrontal supernodal Cholesky (FP64) and the task-queue
// shift-invert solve.  See multifrontal.cuh for the storage scheme.
//
// Factorization of one tree level.  Fronts of at most 32 rows are done by
// one warp each (mf_tiny_front).  Larger fronts are assembled on 32 x 32
// tiles and factored on 64 x 64 tiles (pivot tiles first, then the tiles of
// the rows below the pivots), every tile product on the FP64 tensor cores:
//   assemble  F = A(pivot columns) + shift*I + extend-add of the children's
//             update matrices (pulled per tile, children in a fixed order)
//   for kb:   diag: Cholesky + inverse of the diagonal tile kb (inv into
//             G); rows: the tiles below it as L_Ik = F_Ik inv(L_kk)^T;
//             update of column block kb+1, then of the other trailing
//             tiles, update matrix included.  diag and rows run on a
//             high-priority second branch of the factor graph, so the
//             diagonal step kb+1 overlaps the rest of update kb.
//   invert    the off-diagonal tiles of inv(L11) by recursive doubling
//   wmul      G's lower part = L21 * inv(L11)
// A pivot that is not positive records the failing column in a device status
// word (never a trap); later kernels of the same factorization return early.
#include "multifrontal.cuh"
#include "../common.cuh"
#include "../counters.h"
#include "../host/parallel.h"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

#include <algorithm>
#include <cstring>
#include <new>

#include <type_traits>

#include "../../../include/speigs.h"

// Storage type of the fronts and panels; this file is compiled once for
// double (plain FP64 operator) and once for float (mixed precision).
#ifndef SPX_REAL
#define SPX_REAL double
#endif

namespace spx {

using Real = SPX_REAL;
// G panels: leading dimension and offsets in multiples of 16 bytes, the
// granularity of the bulk copies that stage them in the solve
constexpr int kLdgA = (int)(16 / sizeof(Real));

// memory pool of the device (engine.cu): allocations are cached across calls
cudaMemPool_t device_pool(int dev);

namespace {

constexpr int T = kTile;
constexpr int kFThreads = 256;

struct Sym {
    const int32_t *sfirst, *rows, *relmap, *child_ptr, *child_list;
    const int64_t *rowptr, *frontptr, *gptr;
    // per child: for each 32-row tile boundary of its parent, the first
    // entry of the child's update rows that maps at or below it
    const int32_t *cbnd;
    const int64_t *cbnd_ptr;
};

struct Front {
    int64_t fptr, gptr;
    int r, c, nkb, nt, first;
    int ldg;          // leading dimension of the G panel: r rounded up to 16 bytes
};

// Front geometry with tiles of TS rows/columns: pivot tiles first, then the
// tiles of the rows below the pivots.
template <int TS>
SPX_DEV Front front_of(const Sym &y, int s) {
    Front f;
    f.first = y.sfirst[s];
    f.c = y.sfirst[s + 1] - f.first;
    f.r = (int)(y.rowptr[s + 1] - y.rowptr[s]);
    f.nkb = (f.c + TS - 1) / TS;
    f.nt = f.nkb + (f.r - f.c + TS - 1) / TS;
    f.fptr = y.frontptr[s];
    f.gptr = y.gptr[s];
    f.ldg = (f.r + kLdgA - 1) & ~(kLdgA - 1);
    return f;
}

template <int TS>
SPX_DEV void tile_range(const Front &f, int I, int &a, int &b) {
    if (I < f.nkb) { a = I * TS; b = min(a + TS, f.c); }
    else { a = f.c + (I - f.nkb) * TS; b = min(a + TS, f.r); }
}

// ------------------------------------------------------------ assemble --
__global__ void __launch_bounds__(kFThreads)
mf_assemble(const int4 *__restrict__ tasks, Sym y, Real *__restrict__ F,
            const int32_t *__restrict__ acolptr, const int32_t *__restrict__ atpos,
            const int32_t *__restrict__ asrc, const double *__restrict__ val,
            const double *__restrict__ params, const int *status) {
    __shared__ double S[T][T + 1];
    if (*(volatile const int *)status) return;
    const double shift = params[0];
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z;
    const Front f = front_of<T>(y, s);
    int ra, rb, ca, cb;
    tile_range<T>(f, I, ra, rb);
    tile_range<T>(f, J, ca, cb);
    const int h = rb - ra, w = cb - ca;
    // The children's geometry is read by one thread per child, a batch of
    // kFThreads children at a time, and the children that touch this tile
    // are listed in child order; only those are added, one after another
    // (a parent entry can receive several children's terms, and the fixed
    // order keeps the sums reproducible).
    __shared__ int s_ch[kFThreads], s_ia[kFThreads], s_ja[kFThreads], s_hw[kFThreads];
    __shared__ int s_cnt;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) S[t & (T - 1)][t >> 5] = 0.0;
    const int q0 = y.child_ptr[s], q1 = y.child_ptr[s + 1];
    for (int qb = q0; qb < q1; qb += kFThreads) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        const int q = qb + (int)threadIdx.x;
        int ch = -1, ia = 0, ja = 0, hi = 0, wj = 0;
        if (q < q1) {
            ch = y.child_list[q];
            const int32_t *bd = y.cbnd + y.cbnd_ptr[ch];
            ia = bd[I];
            hi = bd[I + 1] - ia;
            ja = bd[J];
            wj = bd[J + 1] - ja;
        }
        const bool live = hi > 0 && wj > 0;
        // order-preserving compaction: warp ballots, then the warps' counts
        const unsigned bal = __ballot_sync(0xffffffffu, live);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        __shared__ int s_wcnt[kFThreads / 32];
        if (lane == 0) s_wcnt[wid] = __popc(bal);
        __syncthreads();
        if (live) {
            int pos = __popc(bal & ((1u << lane) - 1u));
            for (int w2 = 0; w2 < wid; w2++) pos += s_wcnt[w2];
            s_ch[pos] = ch;
            s_ia[pos] = ia;
            s_ja[pos] = ja;
            s_hw[pos] = hi | (wj << 16);
        }
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w2 = 0; w2 < kFThreads / 32; w2++) tot += s_wcnt[w2];
            s_cnt = tot;
        }
        __syncthreads();
        const int cnt = s_cnt;
        for (int e = 0; e < cnt; e++) {
            const int c2 = s_ch[e], ia2 = s_ia[e], ja2 = s_ja[e];
            const int hi2 = s_hw[e] & 0xffff, wj2 = s_hw[e] >> 16;
            const int rch = (int)(y.rowptr[c2 + 1] - y.rowptr[c2]);
            const int cch = y.sfirst[c2 + 1] - y.sfirst[c2];
            const int32_t *rm = y.relmap + y.rowptr[c2] + cch;
            const Real *U = F + y.frontptr[c2];
            for (int t = threadIdx.x; t < hi2 * wj2; t += blockDim.x) {
                const int i = ia2 + t % hi2, j = ja2 + t / hi2;
                if (i >= j)
                    S[rm[i] - ra][rm[j] - ca] += U[(int64_t)(cch + i) + (int64_t)(cch + j) * rch];
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (J < f.nkb) {
        if (threadIdx.x < w) {
            const int jj = ca + threadIdx.x;
            const int col = f.first + jj;
            for (int e = acolptr[col]; e < acolptr[col + 1]; e++) {
                const int tp = atpos[e];
                if (tp >= ra && tp < rb) S[tp - ra][threadIdx.x] += val[asrc[e]];
            }
            if (I == J) S[jj - ra][threadIdx.x] += shift;
        }
    }
    __syncthreads();
    Real *Fs = F + f.fptr;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        const int i = t & (T - 1), j = t >> 5;
        if (i < h && j < w) Fs[(int64_t)(ra + i) + (int64_t)(ca + j) * f.r] = (Real)S[i][j];
    }
}

// ------------------------------------------------------ warp Cholesky --
// Shared by the diagonal-tile POTRF and the tiny-front kernel: one warp,
// lane i owns row i of M (n <= 32 rows in shared memory).  The scaled column
// j is published in its own array `col`, so the rank-1 updates read it
// without aliasing the rows being updated.  Factors the first c columns of
// the n x n lower matrix M in place (rows >= c receive L21 and the Schur
// complement) and sets dinv[j] = 1 / L(j, j); a pivot <= pivtol records its
// column in *status and is replaced by 1 so the sweep stays finite.
SPX_DEV void warp_cholesky(double (*M)[T + 1], double *col, double *dinv, int n, int c,
                           double pivtol, int *status, int colbase) {
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < c; j++) {
        if (lane == j) {
            double d = M[j][j];
            if (!(d > pivtol)) {
                atomicCAS(status, 0, colbase + j + 1);
                d = 1.0;
            }
            d = sqrt(d);
            M[j][j] = d;
            dinv[j] = 1.0 / d;
        }
        __syncwarp();
        double lij = 0.0;
        if (lane > j && lane < n) {
            lij = M[lane][j] * dinv[j];
            M[lane][j] = lij;
            col[lane] = lij;
        }
        __syncwarp();
        if (lane > j && lane < n)
            for (int k = j + 1; k <= lane; k++) M[lane][k] -= lij * col[k];
        __syncwarp();
    }
}

// X = inv(L11) for the leading c x c block of M, kept in M's strictly upper
// part: X(i, j) for i > j sits at M[j][i] (lane j computes column j), and
// X(j, j) = dinv[j].  The lower part (L) is left as it is.
SPX_DEV void warp_tri_inverse(double (*M)[T + 1], const double *dinv, int c) {
    const int j = threadIdx.x & 31;
    if (j < c) {
        for (int i = j + 1; i < c; i++) {
            double acc = M[i][j] * dinv[j];
            for (int t2 = j + 1; t2 < i; t2++) acc += M[i][t2] * M[j][t2];
            M[j][i] = -acc * dinv[i];
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------- tiny front --
// A front with at most 32 rows is done by one warp end to end: assembly
// (children's update matrices, then A and the shift), partial Cholesky of its
// c pivots with the Schur complement left in the rows below, the update
// matrix written back for the parent, then X = inv(L11) and W = L21 X into G.
constexpr int kTinyWarps = 4;

__global__ void __launch_bounds__(32 * kTinyWarps)
mf_tiny_front(const int4 *__restrict__ tasks, int ntasks, Sym y, Real *__restrict__ F,
              Real *__restrict__ G, const int32_t *__restrict__ acolptr,
              const int32_t *__restrict__ atpos, const int32_t *__restrict__ asrc,
              const double *__restrict__ val, const double *__restrict__ params, int *status) {
    __shared__ double Ms[kTinyWarps][T][T + 1];
    __shared__ double cols[kTinyWarps][T], dinvs[kTinyWarps][T];
    if (*(volatile int *)status) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int task = blockIdx.x * kTinyWarps + wid;
    if (task >= ntasks) return;
    const double shift = params[0];
    const int s = tasks[task].x;
    const Front f = front_of<T>(y, s);
    const int r = f.r, c = f.c;
    double (*M)[T + 1] = Ms[wid];
    for (int k = 0; k < T; k++) M[lane][k] = 0.0;
    __syncwarp();
    for (int q = y.child_ptr[s]; q < y.child_ptr[s + 1]; q++) {
        const int ch = y.child_list[q];
        const int rch = (int)(y.rowptr[ch + 1] - y.rowptr[ch]);
        const int cch = y.sfirst[ch + 1] - y.sfirst[ch];
        const int nb = rch - cch;
        const int32_t *rm = y.relmap + y.rowptr[ch] + cch;
        const Real *U = F + y.frontptr[ch];
        for (int e = lane; e < nb * nb; e += 32) {
            const int a2 = e % nb, b2 = e / nb;
            if (a2 >= b2) M[rm[a2]][rm[b2]] += U[(int64_t)(cch + a2) + (int64_t)(cch + b2) * rch];
        }
        __syncwarp();
    }
    if (lane < c) {
        const int col = f.first + lane;
        for (int e = acolptr[col]; e < acolptr[col + 1]; e++) M[atpos[e]][lane] += val[asrc[e]];
        M[lane][lane] += shift;
    }
    __syncwarp();
    warp_cholesky(M, cols[wid], dinvs[wid], r, c, params[1], status, f.first);
    // update matrix (rows and columns c..r-1) for the parent's assembly
    Real *Fs = F + f.fptr;
    if (lane >= c && lane < r)
        for (int k = c; k <= lane; k++) Fs[(int64_t)lane + (int64_t)k * r] = (Real)M[lane][k];
    const double *dinv = dinvs[wid];
    warp_tri_inverse(M, dinv, c);
    Real *Gs = G + f.gptr;
    if (lane < c) {
        Gs[(int64_t)lane + (int64_t)lane * f.ldg] = (Real)dinv[lane];
        for (int i = lane + 1; i < c; i++) Gs[(int64_t)i + (int64_t)lane * f.ldg] = (Real)M[lane][i];
    }
    // W = L21 X: lane i >= c owns row i
    if (lane >= c && lane < r) {
        for (int j = 0; j < c; j++) {
            double acc = M[lane][j] * dinv[j];
            for (int t2 = j + 1; t2 < c; t2++) acc += M[lane][t2] * M[j][t2];
            Gs[(int64_t)lane + (int64_t)j * f.ldg] = (Real)acc;
        }
    }
}

// ------------------------------------------------------- factor tiles --
// Fronts with more than 32 rows are factored on 64 x 64 tiles.  Every tile
// product runs on the FP64 tensor cores (mma.sync m8n8k4 f64): a CTA of four
// warps owns one 64 x 64 output tile, each warp a 32 x 32 quarter held as
// 4 x 4 accumulator fragments.  Operand tiles are staged in shared memory
// column-major with a leading dimension of 68 doubles, which makes both the
// fragment reads (8 rows x 4 columns per warp) and the coalesced column
// loads free of bank conflicts.
constexpr int FT = 64;
constexpr int FLD = 68;
constexpr int kGThreads = 128;
constexpr int kFTileDoubles = FT * FLD;
constexpr int kPanelGroup = 4;   // panel tiles of a small front share one block
constexpr size_t kPanelSmem = 4 * sizeof(double) * kFTileDoubles;   // mf_diag64
constexpr size_t kRowsSmem = 3 * sizeof(double) * kFTileDoubles;    // mf_rows64
constexpr size_t kPairSmem = 2 * sizeof(double) * kFTileDoubles;

SPX_DEV void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Tile loads go through cp.async (one element per copy, zero-filled outside
// the h x w block), so all of a thread's 32 element copies are in flight at
// once; cp_wait() completes them and makes them visible to the block.
SPX_DEV void cp_async8(double *dst, const double *src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(src),
                 "r"(valid ? 8 : 0) : "memory");
}
SPX_DEV void cp_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
}
SPX_DEV void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most one committed group (the most recent) is still in flight
SPX_DEV void cp_wait_all_but_last() {
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
}
SPX_DEV void cp_async4(float *dst, const float *src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(saddr), "l"(src),
                 "r"(valid ? 4 : 0) : "memory");
}
// FP32 storage: element (i, j) of a tile is copied asynchronously (4 bytes)
// to a 64 x 65 float staging area at the top of the tile's own storage,
// float offset kStageOff + j * FST + i, and the tile is widened in place
// once the copies are complete (tile_widen).  The staging area starts above
// the FP64 columns 0 .. 31, so only the second half of the widening has to
// wait until every staged float has been read.
constexpr int FST = 65;
constexpr int kStageOff = 2 * kFTileDoubles - FT * FST;
static_assert(kStageOff * 4 >= 32 * FLD * 8, "staging area overlaps the first 32 columns");

// one element of a tile (zero when !valid)
template <class MT>
SPX_DEV void elem_copy(double *s, int i, int j, const MT *src, bool valid) {
    if constexpr (std::is_same<MT, double>::value) cp_async8(s + j * FLD + i, src, valid);
    else cp_async4(reinterpret_cast<float *>(s) + kStageOff + j * FST + i, src, valid);
}

// Widen a staged FP32 tile to FP64 in place (a no-op for FP64 storage).  The
// block's copies must be complete and visible (cp_wait); the caller
// synchronises the block again before the tile is read.
template <class MT>
SPX_DEV void tile_widen(double *s) {
    if constexpr (!std::is_same<MT, double>::value) {
        constexpr int kPer = FT * FT / kGThreads, kHalf = kPer / 2;
        const float *f = reinterpret_cast<const float *>(s) + kStageOff;
        float hi[kHalf];
#pragma unroll
        for (int q = 0; q < kHalf; q++) {
            const int t = threadIdx.x + (q + kHalf) * kGThreads;
            hi[q] = f[(t >> 6) * FST + (t & (FT - 1))];
        }
#pragma unroll
        for (int q = 0; q < kHalf; q++) {
            const int t = threadIdx.x + q * kGThreads;
            s[(t >> 6) * FLD + (t & (FT - 1))] = (double)f[(t >> 6) * FST + (t & (FT - 1))];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kHalf; q++) {
            const int t = threadIdx.x + (q + kHalf) * kGThreads;
            s[(t >> 6) * FLD + (t & (FT - 1))] = (double)hi[q];
        }
    }
}

// complete the block's tile copies and make the tiles a (and b) readable
template <class MT>
SPX_DEV void tiles_ready(double *a, double *b = nullptr) {
    cp_wait();
    if constexpr (!std::is_same<MT, double>::value) {
        tile_widen<MT>(a);
        if (b) tile_widen<MT>(b);
        __syncthreads();
    }
}

// s(i, j) = M(ra + i, ca + j) for i < h, j < w; zero elsewhere in the tile
template <class MT>
SPX_DEV void ftile_load(double *s, const MT *M, int64_t ld, int ra, int h, int ca, int w) {
#pragma unroll 8
    for (int q = 0; q < FT * FT / kGThreads; q++) {
        const int t = threadIdx.x + q * kGThreads;
        const int i = t & (FT - 1), j = t >> 6;
        const bool v = (i < h && j < w);
        elem_copy(s, i, j, v ? M + (int64_t)(ra + i) + (int64_t)(ca + j) * ld : M, v);
    }
}
// s(i, j) = M(ca + j, ra + i): the transpose of the stored block
template <class MT>
SPX_DEV void ftile_load_t(double *s, const MT *M, int64_t ld, int ra, int h, int ca, int w) {
#pragma unroll 8
    for (int q = 0; q < FT * FT / kGThreads; q++) {
        const int t = threadIdx.x + q * kGThreads;
        const int j = t & (FT - 1), i = t >> 6;
        const bool v = (i < h && j < w);
        elem_copy(s, i, j, v ? M + (int64_t)(ca + j) + (int64_t)(ra + i) * ld : M, v);
    }
}
// lower triangle of the w x w block at (a, a); zero elsewhere
template <class MT>
SPX_DEV void ftile_load_lower(double *s, const MT *M, int64_t ld, int a, int w) {
#pragma unroll 8
    for (int q = 0; q < FT * FT / kGThreads; q++) {
        const int t = threadIdx.x + q * kGThreads;
        const int i = t & (FT - 1), j = t >> 6;
        const bool v = (i < w && j <= i);
        elem_copy(s, i, j, v ? M + (int64_t)(a + i) + (int64_t)(a + j) * ld : M, v);
    }
}

using Acc = double[4][4][2];

SPX_DEV void acc_zero(Acc &acc) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
}

// acc += A B^T (BT) or A B, with A a 64 x kw tile (s(i, k) at k*FLD + i) and
// B given as 64 x kw (BT: B(n, k) at k*FLD + n) or kw x 64 (B(k, n) at n*FLD + k).
// Only the fragments that touch the first mh rows / nw columns of the
// output are computed (the rest of the accumulator stays zero).
template <bool BT>
SPX_DEV void warp_mma(Acc &acc, const double *As, const double *Bs, int kw, int mh = FT,
                      int nw = FT) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int wid = threadIdx.x >> 5, m0 = (wid & 1) * 32, n0 = (wid >> 1) * 32;
    if (m0 >= mh || n0 >= nw) return;
    const int mi = min(4, (mh - m0 + 7) >> 3), nj = min(4, (nw - n0 + 7) >> 3);
    for (int k = 0; k < kw; k += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = As[(k + t) * FLD + m0 + 8 * i + g];
#pragma unroll
        for (int j = 0; j < 4; j++)
            b[j] = BT ? Bs[(k + t) * FLD + n0 + 8 * j + g] : Bs[(n0 + 8 * j + g) * FLD + k + t];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (i < mi && j < nj) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

// M(ra + m, ca + n) = alpha * acc(m, n) (+ M when add), for m < h, n < w.
// TRANS stores acc(m, n) at M(ca + n, ra + m) instead.
template <bool TRANS, class MT>
SPX_DEV void acc_store(const Acc &acc, MT *M, int64_t ld, int ra, int h, int ca, int w,
                       double alpha, bool add) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int wid = threadIdx.x >> 5, m0 = (wid & 1) * 32, n0 = (wid >> 1) * 32;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int m = m0 + 8 * i + g, n = n0 + 8 * j + 2 * t + e;
                if (m < h && n < w) {
                    MT *p = TRANS ? M + (int64_t)(ca + n) + (int64_t)(ra + m) * ld
                                  : M + (int64_t)(ra + m) + (int64_t)(ca + n) * ld;
                    *p = (MT)(add ? (double)*p + alpha * acc[i][j][e] : alpha * acc[i][j][e]);
                }
            }
}

// M(ra + m, ca + n) = Cs(m, n) - acc(m, n) for m < h, n < w (Cs: the staged
// output tile, column-major FLD)
template <class MT>
SPX_DEV void acc_sub_store(const Acc &acc, const double *Cs, MT *M, int64_t ld, int ra, int h,
                           int ca, int w) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int wid = threadIdx.x >> 5, m0 = (wid & 1) * 32, n0 = (wid >> 1) * 32;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int m = m0 + 8 * i + g, n = n0 + 8 * j + 2 * t + e;
                if (m < h && n < w)
                    M[(int64_t)(ra + m) + (int64_t)(ca + n) * ld] = (MT)(Cs[n * FLD + m] - acc[i][j][e]);
            }
}

// ---- recursive Cholesky + inverse of a diagonal tile (w <= 64) --------
// chol_inv_rec<N>: L (lower) and X = inv(L) of the leading w x w part of the
// N x N lower matrix D (all column-major, leading dimension FLD), by the 128
// threads of the block, 2 x 2 blocked down to 8 x 8:
//   L00, X00 (recursive); L10 = A10 X00^T; A11 -= L10 L10^T and
//   T = L10 X00 (one phase); L11, X11 (recursive); X10 = -X11 T.
// The sequential chain is one 8 x 8 base case per 8 pivots; everything else
// is small products spread over the block.  Rows/columns >= w of L and X are
// zero except for ones on the diagonal (identity padding), so the products
// need no edge tests.  D is destroyed; `tmp` is a scratch tile (64 x FLD).

// 8 x 8 base case by warp 0, lanes 0..7 holding rows in registers
// (not inlined: one copy of the code serves every call site, which keeps the
// recursion's instruction footprint small)
__device__ __noinline__ void chol_inv8(double *D, double *L, double *X, int w, double pivtol,
                                       int *status,
                       int colbase, bool record) {
    if (threadIdx.x >= 32) return;
    const unsigned full = 0xffffffffu;
    const int i = threadIdx.x & 7;
    const bool act = threadIdx.x < 8;
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = (i < w && k <= i) ? D[k * FLD + i] : (k == i ? 1.0 : 0.0);
    double myr = 1.0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        double d = __shfl_sync(full, a[j], j);
        if (!(d > pivtol)) {
            if (record && act && i == 0 && j < w) atomicCAS(status, 0, colbase + j + 1);
            d = 1.0;
        }
        const double rl = rsqrt(d);
        const double lij = (i > j) ? a[j] * rl : (i == j ? d * rl : 0.0);
        a[j] = lij;
        if (i == j) myr = rl;
#pragma unroll
        for (int k = j + 1; k < 8; k++) {
            const double lkj = __shfl_sync(full, lij, k);
            if (k <= i) a[k] -= lij * lkj;
        }
    }
    double x[8];
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = (c == i) ? myr : 0.0;
#pragma unroll
    for (int t = 0; t < 7; t++) {
#pragma unroll
        for (int c = 0; c <= t; c++) {
            const double xtc = __shfl_sync(full, x[c], t);
            if (i > t) x[c] -= a[t] * xtc;
        }
        if (i == t + 1)
#pragma unroll
            for (int c = 0; c <= t; c++) x[c] *= myr;
    }
    if (act)
#pragma unroll
        for (int k = 0; k < 8; k++) {
            L[k * FLD + i] = a[k];
            X[k * FLD + i] = x[k];
        }
}

// C (h x h) = sum_k A(i, k) B'(k, j) over k < h, for the four small products
// of the recursion; each thread computes h*h/128 (or one) outputs.
// mode 0: C = A B^T (A, B both stored row-index-first, i.e. B(j, k))
// mode 1: C = A B   (B(k, j))
template <int H, int MODE>
__device__ __noinline__ void small_mm(const double *A, const double *B, double *C, double alpha,
                                      bool accumulate) {
    constexpr int NOUT = H * H;
    for (int o = threadIdx.x; o < NOUT; o += blockDim.x) {
        const int i = o % H, j = o / H;
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < H; k++)
            acc += A[k * FLD + i] * (MODE == 0 ? B[k * FLD + j] : B[j * FLD + k]);
        C[j * FLD + i] = accumulate ? C[j * FLD + i] + alpha * acc : alpha * acc;
    }
}

template <int N>
SPX_DEV void chol_inv_rec(double *D, double *L, double *X, double *tmp, int w, double pivtol,
                          int *status, int colbase, bool record) {
    if constexpr (N == 8) {
        chol_inv8(D, L, X, w, pivtol, status, colbase, record);
        __syncthreads();
    } else {
        constexpr int H = N / 2;
        const int w0 = min(w, H), w1 = max(w - H, 0);
        chol_inv_rec<H>(D, L, X, tmp, w0, pivtol, status, colbase, record);
        if (w1 == 0) {
            // nothing left to factor: identity padding for the second half
            for (int t = threadIdx.x; t < H * H; t += blockDim.x) {
                const int i = t % H, j = t / H;
                L[(H + j) * FLD + i] = 0.0;
                X[(H + j) * FLD + i] = 0.0;
                L[j * FLD + H + i] = 0.0;
                X[j * FLD + H + i] = 0.0;
                L[(H + j) * FLD + H + i] = (i == j) ? 1.0 : 0.0;
                X[(H + j) * FLD + H + i] = (i == j) ? 1.0 : 0.0;
            }
            __syncthreads();
            return;
        }
        // off-diagonal blocks of L and X above the diagonal stay zero
        for (int t = threadIdx.x; t < H * H; t += blockDim.x) {
            const int i = t % H, j = t / H;
            L[(H + j) * FLD + i] = 0.0;
            X[(H + j) * FLD + i] = 0.0;
        }
        small_mm<H, 0>(D + H, X, L + H, 1.0, false);               // L10 = A10 X00^T
        __syncthreads();
        small_mm<H, 0>(L + H, L + H, D + H * FLD + H, -1.0, true); // A11 -= L10 L10^T
        small_mm<H, 1>(L + H, X, tmp, 1.0, false);                 // T = L10 X00
        __syncthreads();
        chol_inv_rec<H>(D + H * FLD + H, L + H * FLD + H, X + H * FLD + H, tmp + H * FLD, w1,
                        pivtol, status, colbase + H, record);
        small_mm<H, 1>(X + H * FLD + H, tmp, X + H, -1.0, false);  // X10 = -X11 T
        __syncthreads();
    }
}

// Panel step kb of a front, in two kernels that run on separate streams of
// the factor graph.  mf_diag64 (one block per front, task = (s, kb, 0, 0)):
// Cholesky and inverse of the updated diagonal tile kb; inv(L_kk) goes to G
// (only inv(L_kk) is kept: nothing later reads a diagonal tile of L).  It
// needs only the update of that one tile by step kb-1, so it runs beside the
// rest of that step's trailing update.
__global__ void __launch_bounds__(kGThreads)
mf_diag64(const int4 *__restrict__ tasks, Sym y, Real *__restrict__ F, Real *__restrict__ G,
          const double *__restrict__ params, int *status) {
    extern __shared__ double fsm[];
    double *Ds = fsm, *Ls = fsm + kFTileDoubles, *Xs = fsm + 2 * kFTileDoubles;
    double *Ts = fsm + 3 * kFTileDoubles;
    if (*(volatile int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, kb = tk.y;
    const Front f = front_of<FT>(y, s);
    int ka, kz;
    tile_range<FT>(f, kb, ka, kz);
    const int w = kz - ka;
    ftile_load_lower(Ds, F + f.fptr, f.r, ka, w);
    tiles_ready<Real>(Ds);
    chol_inv_rec<64>(Ds, Ls, Xs, Ts, w, params[1], status, f.first + ka, true);
    Real *Gs = G + f.gptr;
    for (int t = threadIdx.x; t < FT * FT; t += blockDim.x) {
        const int i = t & (FT - 1), j = t >> 6;
        if (i < w && j <= i)
            Gs[(int64_t)(ka + i) + (int64_t)(ka + j) * f.ldg] = (Real)Xs[j * FLD + i];
    }
}

// mf_rows64 (task = (s, I0, nI, kb)): the tiles I0 .. I0+nI-1 below the
// diagonal of column block kb, L_Ik = F_Ik inv(L_kk)^T, with inv(L_kk) read
// back from G.  A large front's tiles get a block each, a small front's
// share one; each tile is loaded while the block works on the one before.
__global__ void __launch_bounds__(kGThreads)
mf_rows64(const int4 *__restrict__ tasks, Sym y, Real *__restrict__ F,
          const Real *__restrict__ G, int *status) {
    extern __shared__ double fsm[];
    double *Xs = fsm, *Ps = fsm + kFTileDoubles, *Ds = fsm + 2 * kFTileDoubles;
    if (*(volatile int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I0 = tk.y, nI = tk.z, kb = tk.w;
    const Front f = front_of<FT>(y, s);
    int ka, kz;
    tile_range<FT>(f, kb, ka, kz);
    const int w = kz - ka;
    Real *Fs = F + f.fptr;
    auto load_tile = [&](double *buf, int I) {
        int ra, rb;
        tile_range<FT>(f, I, ra, rb);
        ftile_load(buf, Fs, f.r, ra, rb - ra, ka, w);
    };
    ftile_load_lower(Xs, G + f.gptr, f.ldg, ka, w);
    load_tile(Ps, I0);
    cp_commit();
    double *cur = Ps, *spare = Ds;
    for (int I = I0; I < I0 + nI; I++) {
        if (I + 1 < I0 + nI) load_tile(spare, I + 1);
        cp_commit();
        cp_wait_all_but_last();      // inv(L_kk) and tile I are in
        if constexpr (!std::is_same<Real, double>::value) {
            if (I == I0) tile_widen<Real>(Xs);
            tile_widen<Real>(cur);
            __syncthreads();
        }
        int ra, rb;
        tile_range<FT>(f, I, ra, rb);
        const int h = rb - ra;
        Acc acc;
        acc_zero(acc);
        warp_mma<true>(acc, cur, Xs, (w + 3) & ~3, h, w);
        acc_store<false>(acc, Fs, f.r, ra, h, ka, w, 1.0, false);
        __syncthreads();
        double *t = cur; cur = spare; spare = t;
    }
}

// ---- FP32 trailing update on the TF32 tensor cores (mixed precision) --
// mma.sync m16n8k8 tf32 with FP32 accumulation; every operand is split into
// a TF32 head and a TF32 tail (x = hi + lo) and the product is taken as
// hi*hi + hi*lo + lo*hi, which keeps FP32 accuracy.  Tiles are FP32 in
// shared memory with a leading dimension of 72 floats (conflict-free
// fragment reads).
constexpr int FLDF = 72;

SPX_DEV void ftile_load_f32(float *s, const float *M, int64_t ld, int ra, int h, int ca, int w) {
#pragma unroll 8
    for (int q = 0; q < FT * FT / kGThreads; q++) {
        const int t = threadIdx.x + q * kGThreads;
        const int i = t & (FT - 1), j = t >> 6;
        const bool v = (i < h && j < w);
        cp_async4(s + j * FLDF + i, v ? M + (int64_t)(ra + i) + (int64_t)(ca + j) * ld : M, v);
    }
}
SPX_DEV uint32_t tf32_of(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
SPX_DEV void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = tf32_of(x);
    lo = tf32_of(x - __uint_as_float(hi));
}
SPX_DEV void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// F_IJ -= L_Ik L_Jk^T on FP32 tiles: warp tile 32 x 32 = 2 x 4 fragments.
// The output tile is staged in Cs with the operands, so the subtraction does
// not wait on global loads after the products.
SPX_DEV void update_tile_f32(float *Fs, int ld, int ra, int h, int ca, int w, int ka, int kw,
                             float *As, float *Bs, float *Cs) {
    ftile_load_f32(As, Fs, ld, ra, h, ka, kw);
    ftile_load_f32(Bs, Fs, ld, ca, w, ka, kw);
    ftile_load_f32(Cs, Fs, ld, ra, h, ca, w);
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int wid = threadIdx.x >> 5, m0 = (wid & 1) * 32, n0 = (wid >> 1) * 32;
    if (m0 >= h || n0 >= w) return;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.f;
    const int kw8 = (kw + 7) & ~7;
    for (int k = 0; k < kw8; k += 8) {
        uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int r = m0 + 16 * i + g;
            split_tf32(As[(k + t) * FLDF + r], ah[i][0], al[i][0]);
            split_tf32(As[(k + t) * FLDF + r + 8], ah[i][1], al[i][1]);
            split_tf32(As[(k + t + 4) * FLDF + r], ah[i][2], al[i][2]);
            split_tf32(As[(k + t + 4) * FLDF + r + 8], ah[i][3], al[i][3]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + 8 * j + g;
            split_tf32(Bs[(k + t) * FLDF + n], bh[j][0], bl[j][0]);
            split_tf32(Bs[(k + t + 4) * FLDF + n], bh[j][1], bl[j][1]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                mma_tf32(acc[i][j], al[i], bh[j]);
                mma_tf32(acc[i][j], ah[i], bl[j]);
                mma_tf32(acc[i][j], ah[i], bh[j]);
            }
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int m = m0 + 16 * i + g + 8 * (e >> 1), n = n0 + 8 * j + 2 * t + (e & 1);
                if (m < h && n < w)
                    Fs[(int64_t)(ra + m) + (int64_t)(ca + n) * ld] = Cs[n * FLDF + m] - acc[i][j][e];
            }
}

// F_IJ -= L_Ik L_Jk^T    task = (s, I, J, kb)
__global__ void __launch_bounds__(kGThreads)
mf_update64(const int4 *__restrict__ tasks, Sym y, Real *__restrict__ F, const int *status) {
    extern __shared__ double fsm[];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z, kb = tk.w;
    const Front f = front_of<FT>(y, s);
    int ra, rb, ca, cb, ka, kz;
    tile_range<FT>(f, I, ra, rb);
    tile_range<FT>(f, J, ca, cb);
    tile_range<FT>(f, kb, ka, kz);
    const int h = rb - ra, w = cb - ca, kw = kz - ka;
    Real *Fs = F + f.fptr;
    if constexpr (std::is_same<Real, float>::value) {
        float *As = reinterpret_cast<float *>(fsm), *Bs = As + FT * FLDF, *Cs = Bs + FT * FLDF;
        update_tile_f32(reinterpret_cast<float *>(Fs), f.r, ra, h, ca, w, ka, kw, As, Bs, Cs);
    } else {
        // the output tile is staged with the operands, so the subtraction
        // does not wait on global loads after the products
        double *As = fsm, *Bs = fsm + kFTileDoubles, *Cs = fsm + 2 * kFTileDoubles;
        ftile_load(As, Fs, f.r, ra, h, ka, kw);
        ftile_load(Bs, Fs, f.r, ca, w, ka, kw);
        ftile_load(Cs, Fs, f.r, ra, h, ca, w);
        cp_wait();
        Acc acc;
        acc_zero(acc);
        warp_mma<true>(acc, As, Bs, (kw + 3) & ~3, h, w);
        acc_sub_store(acc, Cs, Fs, f.r, ra, h, ca, w);
    }
}

// inv(L11) by recursive doubling over tile blocks.  After step l every
// diagonal block of 2^l tiles is inverted; step l joins blocks A = [A0, C0)
// and C = [C0, C1) (C0 = A0 + 2^l) through
//   T = L_CA X_A          (mf_inv_t64: T lands in the unused upper part of F)
//   X_CA = -X_C T         (mf_inv_x64)
// task = (s, i, j, l): output tile (i, j), i in C, j in A.
__global__ void __launch_bounds__(kGThreads)
mf_inv_t64(const int4 *__restrict__ tasks, Sym y, Real *__restrict__ F,
           const Real *__restrict__ G, const int *status) {
    extern __shared__ double fsm[];
    double *As = fsm, *Bs = fsm + kFTileDoubles;
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, i = tk.y, j = tk.z, l = tk.w;
    const Front f = front_of<FT>(y, s);
    const int C0 = (j >> (l + 1) << (l + 1)) + (1 << l);
    int ra, rb, ca, cb;
    tile_range<FT>(f, i, ra, rb);
    tile_range<FT>(f, j, ca, cb);
    const int h = rb - ra, w = cb - ca;
    Real *Fs = F + f.fptr;
    const Real *Gs = G + f.gptr;
    Acc acc;
    acc_zero(acc);
    for (int k = j; k < C0; k++) {
        int ka, kz;
        tile_range<FT>(f, k, ka, kz);
        const int kw = kz - ka;
        ftile_load(As, Fs, f.r, ra, h, ka, kw);      // L_ik
        ftile_load(Bs, Gs, f.ldg, ka, kw, ca, w);    // X_kj
        tiles_ready<Real>(As, Bs);
        warp_mma<false>(acc, As, Bs, (kw + 3) & ~3, h, w);
        __syncthreads();
    }
    // T_ij is kept at tile (j, i) of F: strictly upper, never used otherwise
    acc_store<true>(acc, Fs, f.r, ra, h, ca, w, 1.0, false);
}

__global__ void __launch_bounds__(kGThreads)
mf_inv_x64(const int4 *__restrict__ tasks, Sym y, const Real *__restrict__ F,
           Real *__restrict__ G, const int *status) {
    extern __shared__ double fsm[];
    double *As = fsm, *Bs = fsm + kFTileDoubles;
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, i = tk.y, j = tk.z, l = tk.w;
    const Front f = front_of<FT>(y, s);
    const int C0 = (j >> (l + 1) << (l + 1)) + (1 << l);
    int ra, rb, ca, cb;
    tile_range<FT>(f, i, ra, rb);
    tile_range<FT>(f, j, ca, cb);
    const int h = rb - ra, w = cb - ca;
    const Real *Fs = F + f.fptr;
    Real *Gs = G + f.gptr;
    Acc acc;
    acc_zero(acc);
    for (int k = C0; k <= i; k++) {
        int ka, kz;
        tile_range<FT>(f, k, ka, kz);
        const int kw = kz - ka;
        ftile_load(As, Gs, f.ldg, ra, h, ka, kw);    // X_ik
        ftile_load_t(Bs, Fs, f.r, ka, kw, ca, w);    // T_kj, stored transposed at tile (j, k)
        tiles_ready<Real>(As, Bs);
        warp_mma<false>(acc, As, Bs, (kw + 3) & ~3, h, w);
        __syncthreads();
    }
    acc_store<false>(acc, Gs, f.ldg, ra, h, ca, w, -1.0, false);
}

// W_IJ = sum_{K=J}^{nkb-1} L_IK X_KJ   (I a tile of the rows below the pivots)
__global__ void __launch_bounds__(kGThreads)
mf_wmul64(const int4 *__restrict__ tasks, Sym y, const Real *__restrict__ F,
          Real *__restrict__ G, const int *status) {
    extern __shared__ double fsm[];
    double *As = fsm, *Bs = fsm + kFTileDoubles;
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z;
    const Front f = front_of<FT>(y, s);
    int ra, rb, ca, cb;
    tile_range<FT>(f, I, ra, rb);
    tile_range<FT>(f, J, ca, cb);
    const int h = rb - ra, w = cb - ca;
    const Real *Fs = F + f.fptr;
    Real *Gs = G + f.gptr;
    Acc acc;
    acc_zero(acc);
    for (int k = J; k < f.nkb; k++) {
        int ka, kz;
        tile_range<FT>(f, k, ka, kz);
        const int kw = kz - ka;
        ftile_load(As, Fs, f.r, ra, h, ka, kw);
        ftile_load(Bs, Gs, f.ldg, ka, kw, ca, w);
        tiles_ready<Real>(As, Bs);
        warp_mma<false>(acc, As, Bs, (kw + 3) & ~3, h, w);
        __syncthreads();
    }
    acc_store<false>(acc, Gs, f.ldg, ra, h, ca, w, 1.0, false);
}


// ---------------------------------------------------------------- solve --
// The whole solve pair is one persistent kernel that pulls tasks from an
// atomic queue in a topological order (forward tasks leaves -> root, then
// backward tasks root -> leaves) and waits only for the tasks it depends on:
// a forward task for supernode s waits until all children of s are done, a
// backward task until its parent is done.  There is no grid-wide barrier, so
// independent subtrees overlap.  Every task first loads what does not depend
// on other tasks (its panel tile, index lists, b) and only then waits.
// Waits are bounded: a wait that runs out records an error word and returns.
// Deadlock cannot occur: a task waits only on tasks earlier in the queue,
// which are held by running blocks.
//
// Tasks: up to 8 small supernodes (c <= 32, r <= 128) as a bundle, one per
// warp; a larger supernode as 64 x 64 tiles of its panel G, one block task
// per tile that can hold a nonzero.  A tile writes its partial products to
// scratch; the last tile of a row chunk (forward) or column chunk
// (backward), found with an atomic counter, adds the partials in a fixed
// order, so results are the same on every run.
//
// Forward, supernode s:  f = b(pivots) + children's update vectors (host-built
// gather list per front row, children in a fixed order);
// [x1; r2] = G f(0:c);  yf(pivots) = x1;  u_s = f(c:r) - r2.
// Backward:  x1 = G^T [yf(pivots); -x(rows below)].
constexpr int kSThreads = 256;
constexpr int kSWarps = kSThreads / 32;
constexpr int kST = 64;          // rows per forward task, columns per backward task
constexpr int kStrip = 128;      // columns per forward task, rows per backward task
constexpr int kWarpMaxC = 16;    // warp tasks: c <= 16 ...
constexpr int kWarpMaxR = 128;   // ... and r <= 128
constexpr int kGW = 6;           // gather entries per row staged in shared memory
constexpr int kTinyR = 24;       // thread tasks: leaves with r <= 24 ...
constexpr int kTinyC = 6;        // ... and c <= 6
constexpr long kSpinLimit = 1L << 22;

enum { ST_FWD_BUNDLE = 0, ST_FWD_TILE = 1, ST_BWD_BUNDLE = 2, ST_BWD_TILE = 3, ST_FWD_THREADS = 4,
       ST_BWD_THREADS = 5 };

struct SNode {          // per-supernode solve metadata (64 bytes)
    int4 a;             // first, c, r, ldg
    int4 b;             // parent, completions expected from the children
                        // (forward), row chunks, column chunks
    longlong2 p;        // panel offset, row-list offset
    long long uptr;
    int bwd_expect;     // completions of the parent's backward (of its own
                        // forward, for a root) that the backward waits for
    int nchild;
};

struct STask {
    int4 a;             // kind, s, I, J
    int4 b;             // chunk, bundle offset, bundle size, 0
};

struct SolveArgs {
    const SNode *meta;
    const STask *tasks;
    int ntasks, ns;
    const int32_t *bundle, *perm, *rows, *cptr, *cidx;
    const Real *G;
    double *u, *yf, *x;
    const int32_t *fc_base, *fc_n, *bc_base, *bc_n;
    double *fpart, *bpart;
    int *fcnt, *bcnt;
    int *sync;          // block queue | forward arrivals per parent [ns] | forward warp
                        // queue, then unused [ns] | backward arrivals [ns] | root forward
                        // arrivals [ns] | backward warp queue, then unused [ns] | err
    const STask *wtasks;    // warp tasks: nfw forward, then nbw backward
    int nfw, nbw;
    const double *b;
    double *out;
    const int *skip;    // when set and nonzero: nothing to do
};

// relaxed-free publish: a release atomic orders every write that precedes it
// in causality order -- the caller's own, and those of threads that reached a
// block or warp barrier before it -- ahead of the increment
SPX_DEV void add_release(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

SPX_DEV int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait for *p >= target; gives up (and flags *err) after about a
// second, or at once when another wait has already given up.
SPX_DEV void wait_at_least(const int *p, int target, int *err) {
    if (ld_acquire(p) >= target) return;
    for (long it = 0; it < kSpinLimit; it++) {
        __nanosleep(100);
        if (ld_acquire(p) >= target) return;
        if ((it & 255) == 0 && *(volatile int *)err) return;
    }
    atomicExch(err, 1);
}

// Stage the gather list of front row g: count in *n, first kGW indices in
// idx[0..), the list start in *e0 (for entries past kGW).
SPX_DEV void stage_list(const SolveArgs &a, int64_t g, int *idx, int *n, int *e0) {
    const int b0 = a.cptr[g], b1 = a.cptr[g + 1];
    *n = b1 - b0;
    *e0 = b0;
    const int m = min(b1 - b0, kGW);
    for (int e = 0; e < m; e++) idx[e] = a.cidx[b0 + e];
}
SPX_DEV double sum_list(const SolveArgs &a, const int *idx, int n, int e0) {
    double acc = 0.0;
    const int m = min(n, kGW);
    for (int e = 0; e < m; e++) acc += __ldcg(a.u + idx[e]);
    for (int e = kGW; e < n; e++) acc += __ldcg(a.u + a.cidx[e0 + e]);
    return acc;
}

// true in every thread of the block that holds the chunk's last arrival
SPX_DEV bool last_arrival(int *cnt, int n, int *flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int old;
        asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(cnt) : "memory");
        *flag = (old == n - 1);
        if (*flag) *cnt = 0;          // every arrival for this solve is in
    }
    __syncthreads();
    return *flag;
}

// shared memory of one solve block.  gbuf holds one panel strip, staged by
// bulk asynchronous copies (one per panel column) that complete on `bar`.
struct SolveShared {
    Real gbuf[kStrip * kST];          // forward: 128 cols x 64 rows; backward: 64 x 128
    double part[4][kST];
    double vec[kStrip];               // f segment (forward) or v segment (backward)
    double colsum[kST];
    int idx[kStrip][kGW];             // gather lists of the strip's pivot columns
    int cnt[kStrip], e0[kStrip];
    int idx2[kST][kGW];               // gather lists of the chunk's rows below the pivots
    int cnt2[kST], e02[kST];
    int rowv[kStrip];
    int permv[kST];
    double bsum[kST];
};
struct WarpShared {           // per warp in a bundle: gather lists of <= 128 rows
    int idx[kWarpMaxR][kGW];
    int cnt[kWarpMaxR], e0[kWarpMaxR];
};

// Sum p[j] over the 32 lanes for every j < 16 at once: four exchange steps
// (8 + 4 + 2 + 1 shuffles) leave lanes L and L ^ 16 each holding the half
// sum for j = L & 15; one more exchange completes it.
SPX_DEV double transpose_reduce16(double (&p)[16], int lane) {
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const bool hi = lane & 8;
        const double send = hi ? p[m] : p[m + 8];
        const double keep = hi ? p[m + 8] : p[m];
        p[m] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const bool hi = lane & 4;
        const double send = hi ? p[m] : p[m + 4];
        const double keep = hi ? p[m + 4] : p[m];
        p[m] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
#pragma unroll
    for (int m = 0; m < 2; m++) {
        const bool hi = lane & 2;
        const double send = hi ? p[m] : p[m + 2];
        const double keep = hi ? p[m + 2] : p[m];
        p[m] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    {
        const bool hi = lane & 1;
        const double send = hi ? p[0] : p[1];
        const double keep = hi ? p[1] : p[0];
        p[0] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
    }
    return p[0] + __shfl_xor_sync(0xffffffffu, p[0], 16);
}

// ---- bulk asynchronous copies into shared memory, tracked by an mbarrier
SPX_DEV uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
SPX_DEV void mbar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
SPX_DEV void mbar_expect(unsigned long long *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes) : "memory");
}
// copy `bytes` (a multiple of 16, both addresses 16-byte aligned) global -> shared
SPX_DEV void bulk_load(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
SPX_DEV bool mbar_test(unsigned long long *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// bounded wait for the copies of the current phase; a wait that runs out
// flags *err and then waits again (bounded) for the copies still in flight
SPX_DEV void mbar_wait(unsigned long long *bar, uint32_t parity, int *err) {
    for (long it = 0; it < kSpinLimit; it++)
        if (mbar_test(bar, parity)) return;
    atomicExch(err, 1);
    for (long it = 0; it < kSpinLimit; it++)
        if (mbar_test(bar, parity)) return;
}
SPX_DEV void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Stage columns [j0, j0+ncols) x rows [i0, i0+nrows) of a panel (leading
// dimension ldg, column-major) into buf (column stride `stride` doubles):
// one bulk copy per column, issued by the lanes of warp 0.  nrows is even.
SPX_DEV void stage_panel(Real *buf, int stride, const Real *panel, int ldg, int i0, int nrows,
                         int j0, int ncols, unsigned long long *bar) {
    if (threadIdx.x >= 32) return;
    if (threadIdx.x == 0) mbar_expect(bar, (uint32_t)(ncols * nrows * sizeof(Real)));
    __syncwarp();
    for (int jj = threadIdx.x; jj < ncols; jj += 32)
        bulk_load(buf + (size_t)jj * stride, panel + (int64_t)i0 + (int64_t)(j0 + jj) * ldg,
                  (uint32_t)(nrows * sizeof(Real)), bar);
}

// ---- forward, one tiny leaf supernode (r <= 24, c <= 6) per thread.  A
// leaf has no children, so f is b(pivots); the row and column loops are
// unrolled with predication so all of the thread's loads are in flight at once.
SPX_DEV void fwd_thread(const SolveArgs &a, int s) {
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const Real *Gs = a.G + m.p.x;
    double f[kTinyC];
#pragma unroll
    for (int j = 0; j < kTinyC; j++) f[j] = (j < c) ? a.b[a.perm[first + j]] : 0.0;
#pragma unroll
    for (int i = 0; i < kTinyR; i++) {
        if (i < r) {
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < kTinyC; j++)
                if (j < c) acc += Gs[(int64_t)i + (int64_t)j * ldg] * f[j];
            if (i < c) a.yf[first + i] = acc;
            else a.u[m.uptr + (i - c)] = -acc;
        }
    }
    add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
}

// ---- backward, one tiny leaf supernode per thread
SPX_DEV void bwd_thread(const SolveArgs &a, int s) {
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const Real *Gs = a.G + m.p.x;
    int ri[kTinyR];
#pragma unroll
    for (int i = 0; i < kTinyR; i++) ri[i] = (i >= c && i < r) ? rows[i] : 0;
    wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    double v[kTinyR];
#pragma unroll
    for (int i = 0; i < kTinyR; i++)
        v[i] = (i < r) ? ((i < c) ? __ldcg(a.yf + first + i) : -__ldcg(a.x + ri[i])) : 0.0;
#pragma unroll
    for (int j = 0; j < kTinyC; j++) {
        if (j < c) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < kTinyR; i++)
                if (i < r) acc += Gs[(int64_t)i + (int64_t)j * ldg] * v[i];
            a.x[first + j] = acc;
            a.out[a.perm[first + j]] = acc;
        }
    }
    add_release(bdone + s, 1);
}

// ---- forward, one small supernode per warp.  Row i lives in lane i % 32
// (q = i / 32); the panel values of a lane's rows are read in blocks of 4
// columns before they are used, so loads are not serialised behind the
// column loop.
SPX_DEV void fwd_warp(const SolveArgs &a, int s, WarpShared &w) {
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31;
    const int nq = (r + 31) >> 5;
    double bv = 0.0;
    if (lane < c) bv = a.b[a.perm[first + lane]];
    // tiny panels (r <= 32, c <= 8) are read completely before the wait
    double gt[8];
    const bool tiny = (r <= 32 && c <= 8);
    if (tiny) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            gt[j] = (j < c && lane < r) ? Gs[(int64_t)lane + (int64_t)j * ldg] : 0.0;
    }
    if (nchild > 0)
        for (int i = lane; i < r; i += 32) stage_list(a, g0 + i, w.idx[i], &w.cnt[i], &w.e0[i]);
    __syncwarp();
    if (nchild > 0) {
        if (lane == 0) wait_at_least(fcd + s, expect, err);
        __syncwarp();
    }
    double fj = 0.0;
    if (lane < c) fj = bv + (nchild > 0 ? sum_list(a, w.idx[lane], w.cnt[lane], w.e0[lane]) : 0.0);
    double acc[kWarpMaxR / 32];
#pragma unroll
    for (int q = 0; q < kWarpMaxR / 32; q++) acc[q] = 0.0;
    if (tiny) {
#pragma unroll
        for (int j = 0; j < 8; j++) acc[0] += gt[j] * __shfl_sync(0xffffffffu, fj, j);
    } else {
#pragma unroll
        for (int j = 0; j < kWarpMaxC; j++) {
            const double fb = __shfl_sync(0xffffffffu, fj, j);
#pragma unroll
            for (int q = 0; q < kWarpMaxR / 32; q++) {
                const int i = lane + 32 * q;
                if (j < c && q < nq && i < r) acc[q] += Gs[(int64_t)i + (int64_t)j * ldg] * fb;
            }
        }
    }
    // (the panel is zero above the diagonal of its pivot block, so the
    // products above need no masking)
#pragma unroll
    for (int q = 0; q < kWarpMaxR / 32; q++) {
        const int i = lane + 32 * q;
        if (i >= r) continue;
        if (i < c) a.yf[first + i] = acc[q];
        else a.u[m.uptr + (i - c)] =
            (nchild > 0 ? sum_list(a, w.idx[i], w.cnt[i], w.e0[i]) : 0.0) - acc[q];
    }
    __syncwarp();
    if (lane == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
}

// ---- forward, rows [64 I, 64 I + 64) x a 128-column strip S of a large
// supernode's panel.  The strip is staged into shared memory before the
// dependency wait.
SPX_DEV void fwd_tile(const SolveArgs &a, int s, int I, int S, int chunk, SolveShared &sh,
                      unsigned long long *bar, uint32_t &phase, int *flag) {
    int *const fcd = a.sync + 1, *const fchk = fcd + 3 * a.ns, *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w;
    const int parent = m.b.x, nchild = m.nchild, expect = m.b.y;
    const int64_t g0 = m.p.y;
    const int i0 = I * kST, j0 = S * kStrip;
    const int jn = min(kStrip, c - j0);
    // a multiple of 16 bytes: ldg is, and i0 is a multiple of 64
    const int hcopy = min(kST, ldg - i0);
    stage_panel(sh.gbuf, kST, a.G + m.p.x, ldg, i0, hcopy, j0, jn, bar);
    const int t = threadIdx.x;
    double bv = 0.0;
    if (t < jn) {
        bv = a.b[a.perm[first + j0 + t]];
        if (nchild > 0) stage_list(a, g0 + j0 + t, sh.idx[t], &sh.cnt[t], &sh.e0[t]);
    }
    if (t >= kStrip && t < kStrip + kST) {
        const int tt = t - kStrip, ii = i0 + tt;
        if (nchild > 0 && ii >= c && ii < r) stage_list(a, g0 + ii, sh.idx2[tt], &sh.cnt2[tt], &sh.e02[tt]);
    }
    if (nchild > 0 && t == 0) wait_at_least(fcd + s, expect, err);
    __syncthreads();
    if (t < kStrip) {
        sh.vec[t] = (t < jn) ? bv + (nchild > 0 ? sum_list(a, sh.idx[t], sh.cnt[t], sh.e0[t]) : 0.0)
                             : 0.0;
    } else if (t < kStrip + kST) {
        // the children's contributions to the chunk's rows below the pivots,
        // needed by whichever strip finishes the chunk
        const int tt = t - kStrip, ii = i0 + tt;
        sh.bsum[tt] = (nchild > 0 && ii >= c && ii < r)
                          ? sum_list(a, sh.idx2[tt], sh.cnt2[tt], sh.e02[tt]) : 0.0;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    const int row = t & (kST - 1), grp = t >> 6;
    double acc = 0.0;
    if (row < hcopy)
        for (int jj = grp; jj < jn; jj += 4) acc += sh.gbuf[jj * kST + row] * sh.vec[jj];
    sh.part[grp][row] = acc;
    __syncthreads();
    const int nt = a.fc_n[chunk];
    double own = 0.0;
    if (t < kST) {
        own = (sh.part[0][t] + sh.part[1][t]) + (sh.part[2][t] + sh.part[3][t]);
        if (nt > 1) a.fpart[(int64_t)(a.fc_base[chunk] + S) * kST + t] = own;
    }
    // a row chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.fcnt + chunk, nt, flag)) {
        const int ii = i0 + t;
        if (t < kST && ii < r) {
            double rr = own;
            if (nt > 1) {
                const double *p0 = a.fpart + (int64_t)a.fc_base[chunk] * kST + t;
                rr = 0.0;
                for (int q = 0; q < nt; q++) rr += __ldcg(p0 + (int64_t)q * kST);
            }
            if (ii < c) a.yf[first + ii] = rr;
            else a.u[m.uptr + (ii - c)] = sh.bsum[t] - rr;
        }
        __syncthreads();
        // one completed row chunk: the parent counts every chunk of every child
        if (t == 0) add_release(parent >= 0 ? fcd + parent : fchk + s, 1);
    }
    __syncthreads();
}

// ---- backward, one small supernode per warp: column sums x1_j = sum_i
// G(i, j) v_i, with the panel values of blocks of 4 columns loaded before
// their reductions.
SPX_DEV void bwd_warp(const SolveArgs &a, int s) {
    int *const bdone = a.sync + 1 + 2 * a.ns, *const fchk = bdone + a.ns,
              *const err = a.sync + 1 + 5 * a.ns;
    const SNode m = a.meta[s];
    const int first = m.a.x, c = m.a.y, r = m.a.z, ldg = m.a.w, parent = m.b.x;
    const int32_t *rows = a.rows + m.p.y;
    const Real *Gs = a.G + m.p.x;
    const int lane = threadIdx.x & 31;
    const int nq = (r + 31) >> 5;
    int rv[kWarpMaxR / 32];
#pragma unroll
    for (int q = 0; q < kWarpMaxR / 32; q++) {
        const int i = lane + 32 * q;
        rv[q] = (i >= c && i < r) ? rows[i] : 0;
    }
    const int pj = (lane < c) ? a.perm[first + lane] : 0;
    double gt[8];
    const bool tiny = (r <= 32 && c <= 8);
    if (tiny) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            gt[j] = (j < c && lane < r) ? Gs[(int64_t)lane + (int64_t)j * ldg] : 0.0;
    }
    if (lane == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncwarp();
    double v[kWarpMaxR / 32];
#pragma unroll
    for (int q = 0; q < kWarpMaxR / 32; q++) {
        const int i = lane + 32 * q;
        v[q] = (i < r) ? ((i < c) ? __ldcg(a.yf + first + i) : -__ldcg(a.x + rv[q])) : 0.0;
    }
    // every lane accumulates its rows' products for all 16 columns, then one
    // transposing reduction leaves column j's sum in lanes j and j + 16
    double p[kWarpMaxC];
#pragma unroll
    for (int j = 0; j < kWarpMaxC; j++) p[j] = 0.0;
    if (tiny) {
#pragma unroll
        for (int j = 0; j < 8; j++) p[j] = gt[j] * v[0];
    } else {
#pragma unroll
        for (int q = 0; q < kWarpMaxR / 32; q++) {
            const int i = lane + 32 * q;
            if (q < nq && i < r) {
#pragma unroll
                for (int j = 0; j < kWarpMaxC; j++)
                    if (j < c) p[j] += Gs[(int64_t)i + (int64_t)j * ldg] * v[q];
            }
        }
    }
    const double mine = transpose_reduce16(p, lane);
    if (lane < c) {
        a.x[first + lane] = mine;
        a.out[pj] = mine;
    }
    __syncwarp();
    if (lane == 0) add_release(bdone + s, 1);
}

// ---- backward, columns [64 J, 64 J + 64) x a 128-row strip S of a large
// supernode's panel, staged into shared memory before the dependency wait.
SPX_DEV void bwd_tile(const SolveArgs &a, int s, int J, int S, int chunk, SolveShared &sh,
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
    if (t < kStrip) {
        const int ii = i0 + t;
        sh.rowv[t] = (t < in && ii >= c) ? rows[ii] : 0;
    } else if (t < kStrip + kST) {
        const int tt = t - kStrip;
        sh.permv[tt] = (tt < jn) ? a.perm[first + j0 + tt] : 0;
    }
    if (t == 0) wait_at_least(parent >= 0 ? bdone + parent : fchk + s, m.bwd_expect, err);
    __syncthreads();
    if (t < kStrip) {
        const int ii = i0 + t;
        sh.vec[t] = (t < in) ? ((ii < c) ? __ldcg(a.yf + first + ii) : -__ldcg(a.x + sh.rowv[t]))
                             : 0.0;
    }
    mbar_wait(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    const int lane = t & 31, wid = t >> 5;
    const int nt = a.bc_n[chunk];
    {
        // warp wid owns columns wid + 8k, k < 8; lanes own rows lane + 32q
        double p[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int jj = wid + kSWarps * k;
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < kStrip / 32; q++) {
                const int ii = lane + 32 * q;
                if (jj < jn && ii < hcopy) acc += sh.gbuf[jj * kStrip + ii] * sh.vec[ii];
            }
            p[k] = acc;
        }
        // halve the 8 partial columns across lane bits 2, 1, 0, then finish
        // the sums over lane bits 3 and 4: lane L ends with column k = L & 7
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const bool hi = lane & 4;
            const double send = hi ? p[m] : p[m + 4];
            const double keep = hi ? p[m + 4] : p[m];
            p[m] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const bool hi = lane & 2;
            const double send = hi ? p[m] : p[m + 2];
            const double keep = hi ? p[m + 2] : p[m];
            p[m] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
        {
            const bool hi = lane & 1;
            const double send = hi ? p[0] : p[1];
            const double keep = hi ? p[1] : p[0];
            p[0] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
        }
        double col = p[0] + __shfl_xor_sync(0xffffffffu, p[0], 8);
        col += __shfl_xor_sync(0xffffffffu, col, 16);
        if (lane < 8) {
            const int jj = wid + kSWarps * lane;
            if (jj < jn) {
                if (nt > 1) a.bpart[(int64_t)(a.bc_base[chunk] + (S - (j0 / kStrip))) * kST + jj] = col;
                else sh.colsum[jj] = col;
            }
        }
    }
    if (nt == 1) __syncthreads();
    // a column chunk held by one strip needs no cross-block sum
    if (nt == 1 || last_arrival(a.bcnt + chunk, nt, flag)) {
        const int jj = t;
        if (jj < jn) {
            double rr = sh.colsum[jj];
            if (nt > 1) {
                const double *p0 = a.bpart + (int64_t)a.bc_base[chunk] * kST + jj;
                rr = 0.0;
                for (int q = 0; q < nt; q++) rr += __ldcg(p0 + (int64_t)q * kST);
            }
            a.x[first + j0 + jj] = rr;
            a.out[sh.permv[jj]] = rr;
        }
        __syncthreads();
        // one completed column chunk: the children count every chunk
        if (t == 0) add_release(bdone + s, 1);
    }
    __syncthreads();
}

// Warp tasks of one phase: each warp takes the next task from the phase's
// own counter.  A task is one small supernode (ST_*_BUNDLE with one entry)
// or up to 32 tiny leaves, one per lane (ST_*_THREADS).
SPX_DEV void solve_warp_tasks(const SolveArgs &a, const STask *tq, int nt, int *ctr,
                              WarpShared &w) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(ctr, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nt) break;
        const STask tk = tq[t];
        switch (tk.a.x) {
            case ST_FWD_BUNDLE: fwd_warp(a, a.bundle[tk.b.y], w); break;
            case ST_BWD_BUNDLE: bwd_warp(a, a.bundle[tk.b.y]); break;
            case ST_FWD_THREADS:
                if (lane < tk.b.z) fwd_thread(a, a.bundle[tk.b.y + lane]);
                break;
            default:
                if (lane < tk.b.z) bwd_thread(a, a.bundle[tk.b.y + lane]);
                break;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kSThreads, 2) mf_solve_sf(SolveArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int s_task, s_flag;
    __shared__ __align__(8) unsigned long long s_bar;
    SolveShared &sh = *reinterpret_cast<SolveShared *>(smem_raw);
    WarpShared *ws = reinterpret_cast<WarpShared *>(smem_raw);
    if (a.skip && *(volatile const int *)a.skip) return;
    const int wid = threadIdx.x >> 5;
    uint32_t phase = 0;
    if (threadIdx.x == 0) mbar_init(&s_bar);
    // forward warp tasks (the small subtrees), every warp on its own
    solve_warp_tasks(a, a.wtasks, a.nfw, a.sync + 1 + a.ns, ws[wid]);
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
                if (wid < tk.b.z) fwd_warp(a, a.bundle[tk.b.y + wid], ws[wid]);
                break;
            case ST_FWD_TILE:
                fwd_tile(a, tk.a.y, tk.a.z, tk.a.w, tk.b.x, sh, &s_bar, phase, &s_flag);
                break;
            case ST_BWD_BUNDLE:
                if (wid < tk.b.z) bwd_warp(a, a.bundle[tk.b.y + wid]);
                break;
            case ST_FWD_THREADS:
                if ((int)threadIdx.x < tk.b.z) fwd_thread(a, a.bundle[tk.b.y + threadIdx.x]);
                break;
            case ST_BWD_THREADS:
                if ((int)threadIdx.x < tk.b.z) bwd_thread(a, a.bundle[tk.b.y + threadIdx.x]);
                break;
            default:
                bwd_tile(a, tk.a.y, tk.a.z, tk.a.w, tk.b.x, sh, &s_bar, phase, &s_flag);
                break;
        }
        __syncthreads();
        // shared memory read by this task may be refilled by the async
        // proxy in the next one
        fence_proxy_async();
    }
    // backward warp tasks
    solve_warp_tasks(a, a.wtasks + a.nfw, a.nbw, a.sync + 1 + 4 * a.ns, ws[wid]);
}

#include "mf_block_solve.cuh"

static size_t solve_smem_bytes() {
    return std::max(sizeof(SolveShared), sizeof(WarpShared) * kSWarps);
}

// host mirrors of SNode / STask
struct SNodeH {
    int first, c, r, ldg, parent, fwd_expect, nrc, ncc;
    long long gptr, g0, uptr;
    int bwd_expect, nchild;
};
struct STaskH {
    int kind, s, I, J, chunk, boff, bn, pad;
};

template <class Tp>
static int dmalloc(Tp **p, size_t cnt, cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool = device_pool(dev);
    const size_t bytes = (cnt ? cnt : 1) * sizeof(Tp);
    cudaError_t e = pool ? cudaMallocFromPoolAsync((void **)p, bytes, pool, st)
                         : cudaMallocAsync((void **)p, bytes, st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return SPEIGS_ERR_MEM;
    }
    return 0;
}
template <class Tp>
static int dupload(Tp **p, const Tp *h, size_t cnt, cudaStream_t st) {
    int rc = dmalloc(p, cnt, st);
    if (rc) return rc;
    if (cnt) {
        cudaMemcpyAsync(*p, h, cnt * sizeof(Tp), cudaMemcpyHostToDevice, st);
        note_h2d((long long)(cnt * sizeof(Tp)));
    }
    return 0;
}

}  // namespace

template <> MultifrontalPlanT<Real>::~MultifrontalPlanT() { release(0); }

template <> void MultifrontalPlanT<Real>::release(cudaStream_t st) {
    if (fgraph_) { cudaGraphExecDestroy(fgraph_); fgraph_ = nullptr; }
    fgraph_val_ = nullptr;
    direct_val_ = nullptr;
    for (auto &e : fev_)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    if (fside_) { cudaStreamDestroy(fside_); fside_ = nullptr; }
    if (d_params_) { cudaFreeAsync(d_params_, st); d_params_ = nullptr; }
    void *ptrs[] = {d_cbnd_, d_cbnd_ptr_, d_perm_, d_sfirst_, d_rows_, d_relmap_, d_child_ptr_, d_child_list_,
                    d_rowptr_, d_frontptr_, d_gptr_, d_uptr_, d_acolptr_, d_atpos_, d_asrc_,
                    d_tasks_, d_front_, d_G_, d_u_, d_yf_, d_x_, d_status_, d_meta_,
                    d_stask_, d_bundle_, d_cptr_, d_cidx_, d_chunks_, d_fpart_, d_bpart_,
                    d_cnt_, d_sync_, d_byf_, d_bx_, d_bu_, d_bfp_, d_bbp_};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, st);
    d_byf_ = d_bx_ = d_bu_ = d_bfp_ = d_bbp_ = nullptr;
    bw_ = 0;
    d_perm_ = d_sfirst_ = d_rows_ = d_relmap_ = d_child_ptr_ = d_child_list_ = nullptr;
    d_cbnd_ = nullptr;
    d_cbnd_ptr_ = nullptr;
    d_rowptr_ = d_frontptr_ = d_gptr_ = d_uptr_ = nullptr;
    d_acolptr_ = d_atpos_ = d_asrc_ = nullptr;
    d_tasks_ = nullptr;
    d_bundle_ = d_cptr_ = d_cidx_ = d_chunks_ = nullptr;
    d_meta_ = nullptr;
    d_stask_ = nullptr;
    d_fpart_ = d_bpart_ = nullptr;
    d_cnt_ = d_sync_ = nullptr;
    d_front_ = nullptr;
    d_G_ = nullptr;
    d_u_ = d_yf_ = d_x_ = nullptr;
    d_status_ = nullptr;
}

template <> int64_t MultifrontalPlanT<Real>::solve_bytes() const {
    // G read once forward and once backward (lower triangle of the pivot
    // block plus the rows below), the row lists read twice, and the
    // right-hand side, the intermediate and the result vectors.
    return 2 * ((int64_t)sizeof(Real) * g_total_ + 4 * nrows_total_) + 24 * (int64_t)n_;
}

template <> int MultifrontalPlanT<Real>::init(const spx_symbolic &S, const int64_t *rowptr, const int32_t *col,
                           cudaStream_t st) {
    n_ = S.n;
    ns_ = S.nsuper;
    nlevels_ = S.nlevels;
    flops_ = S.flops;
    front_total_ = S.front_total;
    max_rows_ = S.max_rows;
    nrows_total_ = S.rowptr[ns_];
    const int32_t n = n_, ns = ns_;
    try {
        std::vector<int64_t> gptr(ns + 1, 0), uptr(ns + 1, 0);
        int64_t gtri = 0;
        for (int32_t s = 0; s < ns; s++) {
            int64_t r = S.rowptr[s + 1] - S.rowptr[s], c = S.sfirst[s + 1] - S.sfirst[s];
            gptr[s + 1] = gptr[s] + ((r + kLdgA - 1) & ~(int64_t)(kLdgA - 1)) * c;
            uptr[s + 1] = uptr[s] + (r - c);
            gtri += c * (c + 1) / 2 + (r - c) * c;
        }
        g_total_ = gtri;
        u_total_ = uptr[ns];
        // The assembly entries, the solve gather lists and the child tile
        // bounds are independent of the task lists: they are built on side
        // threads while this thread builds the factor and solve task lists.
        std::vector<int32_t> acolptr(n + 1, 0);
        std::vector<int32_t> atpos, asrc;
        std::vector<int32_t> cptr(nrows_total_ + 1, 0), cidx;
        std::vector<int64_t> cbnd_ptr(ns + 1, 0);
        std::vector<int32_t> cbnd;
        TaskGroup side(rowptr[n] >= (1 << 17));
        side.run([&] {
            // assembly entries: for new column j, the entries of A's column
            // perm[j] with new row index >= j, as (row position in the front,
            // index into the CSR values), sorted by row position
            // (counted per column first, so that ranges of supernodes fill
            // their own columns' slices in parallel)
            parallel_ranges(n, 16384, [&](int64_t lo, int64_t hi) {
                for (int64_t j = lo; j < hi; j++) {
                    const int32_t o = S.perm[j];
                    int32_t c = 0;
                    for (int64_t p = rowptr[o]; p < rowptr[o + 1]; p++) c += S.iperm[col[p]] >= j;
                    acolptr[j + 1] = c;
                }
            });
            for (int32_t j = 0; j < n; j++) acolptr[j + 1] += acolptr[j];
            atpos.resize(acolptr[n]);
            asrc.resize(acolptr[n]);
            parallel_ranges(ns, 2048, [&](int64_t lo, int64_t hi) {
                std::vector<int32_t> pos(n, -1);
                std::vector<std::pair<int32_t, int32_t>> tmp;
                for (int64_t s = lo; s < hi; s++) {
                    const int64_t r0 = S.rowptr[s], r1 = S.rowptr[s + 1];
                    for (int64_t t = r0; t < r1; t++) pos[S.rows[t]] = (int32_t)(t - r0);
                    for (int32_t j = S.sfirst[s]; j < S.sfirst[s + 1]; j++) {
                        const int32_t o = S.perm[j];
                        tmp.clear();
                        for (int64_t p = rowptr[o]; p < rowptr[o + 1]; p++) {
                            const int32_t i = S.iperm[col[p]];
                            if (i < j) continue;
                            tmp.emplace_back(pos[i], (int32_t)p);
                        }
                        std::sort(tmp.begin(), tmp.end());
                        int32_t d = acolptr[j];
                        for (auto &e : tmp) { atpos[d] = e.first; asrc[d] = e.second; d++; }
                    }
                    for (int64_t t = r0; t < r1; t++) pos[S.rows[t]] = -1;
                }
            });
        });
        side.run([&] {
            // gather lists: for every front row (global row-list index g) the
            // update-vector entries of the children that land on it, children in
            // their fixed order
            for (int32_t par = 0; par < ns; par++)
                for (int32_t q = S.child_ptr[par]; q < S.child_ptr[par + 1]; q++) {
                    const int ch = S.child_list[q];
                    const int cc = S.sfirst[ch + 1] - S.sfirst[ch];
                    for (int64_t t = S.rowptr[ch] + cc; t < S.rowptr[ch + 1]; t++)
                        cptr[S.rowptr[par] + S.relmap[t] + 1]++;
                }
            for (int64_t g = 0; g < nrows_total_; g++) cptr[g + 1] += cptr[g];
            cidx.assign(cptr[nrows_total_], 0);
            {
                std::vector<int32_t> fill(cptr.begin(), cptr.end() - 1);
                for (int32_t par = 0; par < ns; par++)
                    for (int32_t q = S.child_ptr[par]; q < S.child_ptr[par + 1]; q++) {
                        const int ch = S.child_list[q];
                        const int cc = S.sfirst[ch + 1] - S.sfirst[ch];
                        for (int64_t t = S.rowptr[ch] + cc; t < S.rowptr[ch + 1]; t++)
                            cidx[fill[S.rowptr[par] + S.relmap[t]]++] =
                                (int32_t)(uptr[ch] + (t - S.rowptr[ch] - cc));
                    }
            }
        });
        side.run([&] {
            // child tile bounds for the assembly (32-row tiles of the parent)
            for (int32_t ch = 0; ch < ns; ch++) {
                const int p = S.sparent[ch];
                cbnd_ptr[ch] = (int64_t)cbnd.size();
                if (p < 0) continue;
                const int rp = (int)(S.rowptr[p + 1] - S.rowptr[p]);
                const int cp = S.sfirst[p + 1] - S.sfirst[p];
                const int nkb = (cp + T - 1) / T, ntp = nkb + (rp - cp + T - 1) / T;
                const int cch = S.sfirst[ch + 1] - S.sfirst[ch];
                const int32_t *rm = S.relmap + S.rowptr[ch] + cch;
                const int nb = (int)(S.rowptr[ch + 1] - S.rowptr[ch]) - cch;
                for (int I = 0; I <= ntp; I++) {
                    const int start = (I == ntp) ? rp : (I < nkb ? I * T : cp + (I - nkb) * T);
                    cbnd.push_back((int32_t)(std::lower_bound(rm, rm + nb, start) - rm));
                }
            }
            cbnd_ptr[ns] = (int64_t)cbnd.size();
        });
        // tile task lists, level by level (on a side thread: nothing below
        // reads them before the uploads)
        std::vector<int4> tasks;
        side.run([&] {
            launches_.clear();
            use_side_ = false;
            auto emit = [&](int kind, size_t before) {
                if (tasks.size() > before)
                    launches_.push_back({kind, (int64_t)before, (int64_t)(tasks.size() - before)});
            };
            auto is_tiny = [&](int s) { return S.rowptr[s + 1] - S.rowptr[s] <= T; };
            for (int l = 0; l < S.nlevels; l++) {
                const int32_t q0 = S.level_ptr[l], q1 = S.level_ptr[l + 1];
                int nkbmax = 0;
                {
                    size_t bt = tasks.size();
                    for (int32_t q = q0; q < q1; q++)
                        if (is_tiny(S.level_sup[q])) tasks.push_back(make_int4(S.level_sup[q], 0, 0, 0));
                    emit(MF_TINY, bt);
                }
                size_t b = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    if (is_tiny(s)) continue;
                    const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                    const int c = S.sfirst[s + 1] - S.sfirst[s];
                    const int nkb = (c + T - 1) / T, nt = nkb + (r - c + T - 1) / T;
                    nkbmax = std::max(nkbmax, nkb);
                    for (int I = 0; I < nt; I++)
                        for (int J = 0; J <= I; J++) tasks.push_back(make_int4(s, I, J, 0));
                }
                emit(MF_ASSEMBLE, b);
                // factor steps on 64-tiles: diagonal tile kb, the tiles below
                // it, then the right-looking update of the trailing tiles,
                // Schur complement included
                auto geo = [&](int s, int &r, int &c, int &nkb, int &nt) {
                    r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                    c = S.sfirst[s + 1] - S.sfirst[s];
                    nkb = (c + FT - 1) / FT;
                    nt = nkb + (r - c + FT - 1) / FT;
                };
                nkbmax = 0;
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    if (is_tiny(s)) continue;
                    int r, c, nkb, nt;
                    geo(s, r, c, nkb, nt);
                    nkbmax = std::max(nkbmax, nkb);
                }
                // step kb: the diagonal tile (mf_diag64), the tiles below it
                // (mf_rows64), the update of column block kb+1 (the next
                // diagonal tile depends only on it), then the rest of the
                // trailing update, which runs beside the next diagonal step.
                // These four launches are recorded even when empty: they carry
                // the cross-stream ordering of the factor graph.
                auto emit_always = [&](int kind, size_t before) {
                    launches_.push_back({kind, (int64_t)before, (int64_t)(tasks.size() - before)});
                };
                if (nkbmax >= 2) use_side_ = true;
                for (int kb = 0; kb < nkbmax; kb++) {
                    size_t b0 = tasks.size();
                    for (int32_t q = q0; q < q1; q++) {
                        const int s = S.level_sup[q];
                        if (is_tiny(s)) continue;
                        int r, c, nkb, nt;
                        geo(s, r, c, nkb, nt);
                        if (nkb > kb) tasks.push_back(make_int4(s, kb, 0, 0));
                    }
                    emit_always(MF_DIAG, b0);
                    b0 = tasks.size();
                    for (int32_t q = q0; q < q1; q++) {
                        const int s = S.level_sup[q];
                        if (is_tiny(s)) continue;
                        int r, c, nkb, nt;
                        geo(s, r, c, nkb, nt);
                        if (nkb <= kb || nt - kb <= 1) continue;
                        // a front with few tiles left: one block; else one per tile
                        if (nt - kb - 1 <= kPanelGroup) tasks.push_back(make_int4(s, kb + 1, nt - kb - 1, kb));
                        else
                            for (int I = kb + 1; I < nt; I++) tasks.push_back(make_int4(s, I, 1, kb));
                    }
                    emit_always(MF_ROWS, b0);
                    b0 = tasks.size();
                    for (int32_t q = q0; q < q1; q++) {
                        const int s = S.level_sup[q];
                        if (is_tiny(s)) continue;
                        int r, c, nkb, nt;
                        geo(s, r, c, nkb, nt);
                        if (nkb <= kb) continue;
                        for (int I = kb + 1; I < nt; I++) tasks.push_back(make_int4(s, I, kb + 1, kb));
                    }
                    emit_always(MF_UPD_NEXT, b0);
                    b0 = tasks.size();
                    for (int32_t q = q0; q < q1; q++) {
                        const int s = S.level_sup[q];
                        if (is_tiny(s)) continue;
                        int r, c, nkb, nt;
                        geo(s, r, c, nkb, nt);
                        if (nkb <= kb) continue;
                        for (int I = kb + 2; I < nt; I++)
                            for (int J = kb + 2; J <= I; J++) tasks.push_back(make_int4(s, I, J, kb));
                    }
                    emit(MF_UPDATE, b0);
                }
                for (int l = 0; (1 << l) < nkbmax; l++) {
                    const int half = 1 << l;
                    for (int phase = 0; phase < 2; phase++) {
                        size_t b0 = tasks.size();
                        for (int32_t q = q0; q < q1; q++) {
                            const int s = S.level_sup[q];
                            if (is_tiny(s)) continue;
                            int r, c, nkb, nt;
                            geo(s, r, c, nkb, nt);
                            for (int A0 = 0; A0 + half < nkb; A0 += 2 * half) {
                                const int C0 = A0 + half, C1 = std::min(A0 + 2 * half, nkb);
                                for (int i = C0; i < C1; i++)
                                    for (int j = A0; j < C0; j++) tasks.push_back(make_int4(s, i, j, l));
                            }
                        }
                        emit(phase == 0 ? MF_INV_T : MF_INV_X, b0);
                    }
                }
                size_t bw = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    if (is_tiny(s)) continue;
                    int r, c, nkb, nt;
                    geo(s, r, c, nkb, nt);
                    for (int I = nkb; I < nt; I++)
                        for (int J = 0; J < nkb; J++) tasks.push_back(make_int4(s, I, J, 0));
                }
                emit(MF_WMUL, bw);
            }
        });
        // solve: per-supernode metadata and the task queue.  Forward tasks
        // level by level from the leaves (tiles of large supernodes first,
        // then bundles of up to 8 small ones), then backward tasks level by
        // level from the roots.  Every task depends only on earlier tasks.
        std::vector<SNodeH> meta(ns);
        auto small = [&](int r, int c) { return c <= kWarpMaxC && r <= kWarpMaxR; };
        std::vector<STaskH> tasks_s;
        std::vector<int32_t> bundle, fc_base, fc_n, bc_base, bc_n;
        int32_t fslots = 0, bslots = 0;
        // one thread per tiny leaf; everything else small goes to a warp
        auto tiny_leaf = [&](int s2) {
            return meta[s2].c <= kTinyC && meta[s2].r <= kTinyR && meta[s2].nchild == 0;
        };
        for (int32_t s2 = 0; s2 < ns; s2++) {
            const int r = (int)(S.rowptr[s2 + 1] - S.rowptr[s2]);
            const int c = S.sfirst[s2 + 1] - S.sfirst[s2];
            SNodeH &m = meta[s2];
            m.first = S.sfirst[s2]; m.c = c; m.r = r; m.ldg = (r + kLdgA - 1) & ~(kLdgA - 1);
            m.parent = S.sparent[s2];
            m.nchild = S.child_ptr[s2 + 1] - S.child_ptr[s2];
            m.nrc = (r + kST - 1) / kST;
            m.ncc = (c + kST - 1) / kST;
            m.gptr = gptr[s2]; m.g0 = S.rowptr[s2]; m.uptr = uptr[s2];
            m.fwd_expect = 0;
            m.bwd_expect = 0;
        }
        // completions a supernode reports: one per row chunk (forward) or
        // column chunk (backward) when it is cut into tiles, else one
        auto fwd_done_count = [&](int s2) {
            return small(meta[s2].r, meta[s2].c) ? 1 : meta[s2].nrc;
        };
        auto bwd_done_count = [&](int s2) {
            return small(meta[s2].r, meta[s2].c) ? 1 : meta[s2].ncc;
        };
        for (int32_t s2 = 0; s2 < ns; s2++) {
            const int p2 = meta[s2].parent;
            if (p2 >= 0) {
                meta[p2].fwd_expect += fwd_done_count(s2);
                meta[s2].bwd_expect = bwd_done_count(p2);
            } else {
                meta[s2].bwd_expect = fwd_done_count(s2);
            }
        }
        // The small supernodes of a level are bundled by decreasing work (rows
        // per lane, then pivots): a bundle's warps then finish together, and
        // the longest bundles are dequeued first.  Supernodes of one level do
        // not depend on each other, and each is computed the same way in any
        // bundle, so the results do not change.
        auto sort_by_work = [&](std::vector<int32_t> &v) {
            std::stable_sort(v.begin(), v.end(), [&](int32_t x, int32_t y2) {
                const int qx = (meta[x].r + 31) / 32, qy = (meta[y2].r + 31) / 32;
                if (qx != qy) return qx > qy;
                return meta[x].c > meta[y2].c;
            });
        };
        // Warp tasks: a small supernode whose whole subtree is small is solved
        // by one warp that dequeues it on its own (a tiny leaf by one lane of
        // a warp, 32 to a task), in a phase before (forward) or after
        // (backward) the block tasks.  A warp task then never waits for a
        // block task in the forward pass, and no block task waits for a warp
        // task of the backward pass, so neither phase can stall the other.
        std::vector<char> warpable(ns, 0);
        for (int l = 0; l < S.nlevels; l++)
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                bool ok = small(meta[s2].r, meta[s2].c);
                for (int32_t e = S.child_ptr[s2]; ok && e < S.child_ptr[s2 + 1]; e++)
                    ok = warpable[S.child_list[e]] != 0;
                warpable[s2] = ok;
            }
        std::vector<STaskH> wtasks_f, wtasks_b;
        auto emit_warp_level = [&](int l, bool fwd) {
            std::vector<int32_t> sm, ti;
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                if (!warpable[s2]) continue;
                if (tiny_leaf(s2)) ti.push_back(s2);
                else sm.push_back(s2);
            }
            sort_by_work(sm);
            std::vector<STaskH> &out = fwd ? wtasks_f : wtasks_b;
            for (int32_t s2 : sm) {
                out.push_back({fwd ? ST_FWD_BUNDLE : ST_BWD_BUNDLE, 0, 0, 0, 0,
                               (int)bundle.size(), 1, 0});
                bundle.push_back(s2);
            }
            for (size_t b0 = 0; b0 < ti.size(); b0 += 32) {
                const int nb = (int)std::min<size_t>(32, ti.size() - b0);
                out.push_back({fwd ? ST_FWD_THREADS : ST_BWD_THREADS, 0, 0, 0, 0,
                               (int)bundle.size(), nb, 0});
                bundle.insert(bundle.end(), ti.begin() + b0, ti.begin() + b0 + nb);
            }
        };
        for (int l = 0; l < S.nlevels; l++) emit_warp_level(l, true);
        for (int l = S.nlevels - 1; l >= 0; l--) emit_warp_level(l, false);
        for (int l = 0; l < S.nlevels; l++) {
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                const int r = meta[s2].r, c = meta[s2].c;
                if (small(r, c)) continue;
                const int nI = meta[s2].nrc, nS = (c + kStrip - 1) / kStrip;
                for (int I = 0; I < nI; I++) {
                    // strip S can hold a nonzero of row chunk I iff the chunk's
                    // last row >= the strip's first column
                    const int smax = std::min(nS - 1, (std::min(r, (I + 1) * kST) - 1) / kStrip);
                    const int chunk = (int)fc_base.size();
                    fc_base.push_back(fslots);
                    fc_n.push_back(smax + 1);
                    fslots += smax + 1;
                    for (int S2 = 0; S2 <= smax; S2++)
                        tasks_s.push_back({ST_FWD_TILE, s2, I, S2, chunk, 0, 0, 0});
                }
            }
            std::vector<int32_t> sm, ti;
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                if (warpable[s2]) continue;
                if (tiny_leaf(s2)) ti.push_back(s2);
                else if (small(meta[s2].r, meta[s2].c)) sm.push_back(s2);
            }
            sort_by_work(sm);
            for (size_t b0 = 0; b0 < sm.size(); b0 += kSWarps) {
                const int nb = (int)std::min<size_t>(kSWarps, sm.size() - b0);
                tasks_s.push_back({ST_FWD_BUNDLE, 0, 0, 0, 0, (int)bundle.size(), nb, 0});
                bundle.insert(bundle.end(), sm.begin() + b0, sm.begin() + b0 + nb);
            }
            for (size_t b0 = 0; b0 < ti.size(); b0 += kSThreads) {
                const int nb = (int)std::min<size_t>(kSThreads, ti.size() - b0);
                tasks_s.push_back({ST_FWD_THREADS, 0, 0, 0, 0, (int)bundle.size(), nb, 0});
                bundle.insert(bundle.end(), ti.begin() + b0, ti.begin() + b0 + nb);
            }
        }
        for (int l = S.nlevels - 1; l >= 0; l--) {
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                const int r = meta[s2].r, c = meta[s2].c;
                if (small(r, c)) continue;
                const int nJ = meta[s2].ncc, nS = (r + kStrip - 1) / kStrip;
                for (int J = 0; J < nJ; J++) {
                    // row strips from the one holding the chunk's first column
                    const int smin = (J * kST) / kStrip;
                    const int chunk = (int)bc_base.size();
                    bc_base.push_back(bslots);
                    bc_n.push_back(nS - smin);
                    bslots += nS - smin;
                    for (int S2 = smin; S2 < nS; S2++)
                        tasks_s.push_back({ST_BWD_TILE, s2, J, S2, chunk, 0, 0, 0});
                }
            }
            std::vector<int32_t> sm, ti;
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s2 = S.level_sup[q];
                if (warpable[s2]) continue;
                if (tiny_leaf(s2)) ti.push_back(s2);
                else if (small(meta[s2].r, meta[s2].c)) sm.push_back(s2);
            }
            sort_by_work(sm);
            for (size_t b0 = 0; b0 < sm.size(); b0 += kSWarps) {
                const int nb = (int)std::min<size_t>(kSWarps, sm.size() - b0);
                tasks_s.push_back({ST_BWD_BUNDLE, 0, 0, 0, 0, (int)bundle.size(), nb, 0});
                bundle.insert(bundle.end(), sm.begin() + b0, sm.begin() + b0 + nb);
            }
            for (size_t b0 = 0; b0 < ti.size(); b0 += kSThreads) {
                const int nb = (int)std::min<size_t>(kSThreads, ti.size() - b0);
                tasks_s.push_back({ST_BWD_THREADS, 0, 0, 0, 0, (int)bundle.size(), nb, 0});
                bundle.insert(bundle.end(), ti.begin() + b0, ti.begin() + b0 + nb);
            }
        }
        ntasks_ = (int)tasks_s.size();
        nfw_ = (int)wtasks_f.size();
        nbw_ = (int)wtasks_b.size();
        tasks_s.insert(tasks_s.end(), wtasks_f.begin(), wtasks_f.end());
        tasks_s.insert(tasks_s.end(), wtasks_b.begin(), wtasks_b.end());
        side.wait();
        int rc = 0;
        rc = rc ? rc : dupload(&d_cbnd_, cbnd.data(), cbnd.size(), st);
        rc = rc ? rc : dupload(&d_cbnd_ptr_, cbnd_ptr.data(), cbnd_ptr.size(), st);
        rc = rc ? rc : dupload(&d_perm_, S.perm, n, st);
        rc = rc ? rc : dupload(&d_sfirst_, S.sfirst, ns + 1, st);
        rc = rc ? rc : dupload(&d_rows_, S.rows, (size_t)nrows_total_, st);
        rc = rc ? rc : dupload(&d_relmap_, S.relmap, (size_t)nrows_total_, st);
        rc = rc ? rc : dupload(&d_child_ptr_, S.child_ptr, ns + 1, st);
        rc = rc ? rc : dupload(&d_child_list_, S.child_list, ns, st);
        rc = rc ? rc : dupload(&d_rowptr_, S.rowptr, ns + 1, st);
        rc = rc ? rc : dupload(&d_frontptr_, S.frontptr, ns + 1, st);
        rc = rc ? rc : dupload(&d_gptr_, gptr.data(), ns + 1, st);
        rc = rc ? rc : dupload(&d_uptr_, uptr.data(), ns + 1, st);
        rc = rc ? rc : dupload(&d_acolptr_, acolptr.data(), n + 1, st);
        rc = rc ? rc : dupload(&d_atpos_, atpos.data(), atpos.size(), st);
        rc = rc ? rc : dupload(&d_asrc_, asrc.data(), asrc.size(), st);
        rc = rc ? rc : dupload(&d_tasks_, tasks.data(), tasks.size(), st);
        {
            std::vector<int32_t> ch;
            ch.insert(ch.end(), fc_base.begin(), fc_base.end());
            ch.insert(ch.end(), fc_n.begin(), fc_n.end());
            ch.insert(ch.end(), bc_base.begin(), bc_base.end());
            ch.insert(ch.end(), bc_n.begin(), bc_n.end());
            rc = rc ? rc : dupload(&d_chunks_, ch.data(), ch.size(), st);
            nfc_ = (int32_t)fc_base.size();
            nbc_ = (int32_t)bc_base.size();
        }
        static_assert(sizeof(SNodeH) == sizeof(SNode), "metadata layout");
        static_assert(sizeof(STaskH) == sizeof(STask), "task layout");
        rc = rc ? rc : dupload((SNodeH **)&d_meta_, meta.data(), meta.size(), st);
        rc = rc ? rc : dupload((STaskH **)&d_stask_, tasks_s.data(), tasks_s.size(), st);
        rc = rc ? rc : dupload(&d_bundle_, bundle.data(), bundle.size(), st);
        fslots_ = fslots;
        bslots_ = bslots;
        rc = rc ? rc : dmalloc(&d_fpart_, (size_t)fslots * kST, st);
        rc = rc ? rc : dmalloc(&d_bpart_, (size_t)bslots * kST, st);
        rc = rc ? rc : dmalloc(&d_cnt_, (size_t)(nfc_ + nbc_), st);
        if (!rc) cudaMemsetAsync(d_cnt_, 0, sizeof(int) * (size_t)(nfc_ + nbc_), st);
        sync_ints_ = 2 + 5 * (size_t)ns;
        rc = rc ? rc : dmalloc(&d_sync_, sync_ints_, st);
        if (!rc) cudaMemsetAsync(d_sync_, 0, sizeof(int) * sync_ints_, st);
        rc = rc ? rc : dupload(&d_cptr_, cptr.data(), cptr.size(), st);
        rc = rc ? rc : dupload(&d_cidx_, cidx.data(), cidx.size(), st);
        rc = rc ? rc : dmalloc(&d_G_, (size_t)gptr[ns], st);
        // the solve reads whole tiles: the strictly upper part of every
        // inv(L11) block and the padding row stay zero for the plan's life
        if (!rc) cudaMemsetAsync(d_G_, 0, sizeof(Real) * (size_t)gptr[ns], st);
        rc = rc ? rc : dmalloc(&d_u_, (size_t)u_total_, st);
        rc = rc ? rc : dmalloc(&d_yf_, (size_t)n, st);
        rc = rc ? rc : dmalloc(&d_x_, (size_t)n, st);
        rc = rc ? rc : dmalloc(&d_status_, 1, st);
        if (rc) return rc;
        // everything uploaded above comes from host vectors that die here
        if (cudaStreamSynchronize(st) != cudaSuccess) return SPEIGS_ERR_INTERNAL;
        // persistent grid for the task-queue solve
        // factor tile kernels stage two or three 64 x 64 tiles
        cudaFuncSetAttribute(mf_diag64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem);
        cudaFuncSetAttribute(mf_rows64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRowsSmem);
        cudaFuncSetAttribute(mf_update64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(3 * sizeof(double) * kFTileDoubles));
        cudaFuncSetAttribute(mf_inv_t64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem);
        cudaFuncSetAttribute(mf_inv_x64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem);
        cudaFuncSetAttribute(mf_wmul64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem);
        solve_smem_ = solve_smem_bytes();
        if (solve_smem_ > 48 * 1024)
            cudaFuncSetAttribute(mf_solve_sf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)solve_smem_);
        int dev = 0, nsm = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mf_solve_sf, kSThreads, solve_smem_);
        if (per_sm <= 0 || nsm <= 0) return SPEIGS_ERR_INTERNAL;
        solve_grid_ = nsm * std::min(per_sm, 4);
    } catch (const std::bad_alloc &) {
        return SPEIGS_ERR_MEM;
    }
    return 0;
}

template <> void MultifrontalPlanT<Real>::launch_factor(const double *d_val, cudaStream_t st) {
    Sym y{d_sfirst_, d_rows_, d_relmap_, d_child_ptr_, d_child_list_, d_rowptr_, d_frontptr_,
          d_gptr_, d_cbnd_, d_cbnd_ptr_};
    // with no front of two or more column blocks there is nothing to overlap:
    // every launch goes on st, in order
    const bool side = use_side_ && fside_;
    cudaStream_t sd = side ? fside_ : st;
    for (const MfLaunch &L : launches_) {
        const int4 *tk = d_tasks_ + L.off;
        const unsigned nb = (unsigned)L.count;
        switch (L.kind) {
            case MF_ASSEMBLE:
                mf_assemble<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_acolptr_, d_atpos_,
                                                      d_asrc_, d_val, d_params_, d_status_);
                if (side) cudaEventRecord(fev_[0], st);
                break;
            case MF_TINY:
                mf_tiny_front<<<(nb + kTinyWarps - 1) / kTinyWarps, 32 * kTinyWarps, 0, st>>>(
                    tk, (int)nb, y, d_front_, d_G_, d_acolptr_, d_atpos_, d_asrc_, d_val, d_params_,
                    d_status_);
                break;
            case MF_DIAG:
                // after the update of this diagonal tile (the last record of
                // fev_[0] on st), beside the rest of the previous update
                if (side) cudaStreamWaitEvent(sd, fev_[0], 0);
                if (nb) mf_diag64<<<nb, kGThreads, kPanelSmem, sd>>>(tk, y, d_front_, d_G_,
                                                                      d_params_, d_status_);
                break;
            case MF_ROWS:
                if (nb) mf_rows64<<<nb, kGThreads, kRowsSmem, sd>>>(tk, y, d_front_, d_G_,
                                                                     d_status_);
                if (side) cudaEventRecord(fev_[1], sd);
                break;
            case MF_UPD_NEXT:
                if (side) cudaStreamWaitEvent(st, fev_[1], 0);
                if (nb) mf_update64<<<nb, kGThreads, 3 * sizeof(double) * kFTileDoubles, st>>>(
                    tk, y, d_front_, d_status_);
                if (side) cudaEventRecord(fev_[0], st);
                break;
            case MF_UPDATE:
                mf_update64<<<nb, kGThreads, 3 * sizeof(double) * kFTileDoubles, st>>>(
                    tk, y, d_front_, d_status_);
                break;
            case MF_INV_T:
                mf_inv_t64<<<nb, kGThreads, kPairSmem, st>>>(tk, y, d_front_, d_G_, d_status_);
                break;
            case MF_INV_X:
                mf_inv_x64<<<nb, kGThreads, kPairSmem, st>>>(tk, y, d_front_, d_G_, d_status_);
                break;
            case MF_WMUL:
                mf_wmul64<<<nb, kGThreads, kPairSmem, st>>>(tk, y, d_front_, d_G_, d_status_);
                break;
        }
    }
}

// The launch sequence is fixed by the symbolic analysis, so it is captured
// once into a CUDA graph and replayed; the shift and the pivot tolerance are
// read from device memory by the kernels.
template <> int MultifrontalPlanT<Real>::factorize(const double *d_val, double shift, double pivtol,
                                cudaStream_t st) {
    if (!d_front_) {
        if (dmalloc(&d_front_, (size_t)front_total_, st)) return SPEIGS_ERR_MEM;
    }
    if (!d_params_) {
        if (dmalloc(&d_params_, 2, st)) return SPEIGS_ERR_MEM;
    }
    const double hp[2] = {shift, pivtol};
    cudaMemcpyAsync(d_params_, hp, sizeof hp, cudaMemcpyHostToDevice, st);
    note_h2d(sizeof hp);
    cudaMemsetAsync(d_status_, 0, sizeof(int), st);
    if (use_side_ && !fside_) {
        // the factor graph's second branch (diagonal steps) and its joins;
        // the branch has the highest priority, so its blocks are scheduled
        // ahead of the waiting blocks of a large trailing update
        int prio_lo = 0, prio_hi = 0;
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
        if (cudaStreamCreateWithPriority(&fside_, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
            cudaEventCreateWithFlags(&fev_[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&fev_[1], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return SPEIGS_ERR_INTERNAL;
        }
    }
    bool direct = false;
    if (!fgraph_ || fgraph_val_ != d_val) {
        if (fgraph_) { cudaGraphExecDestroy(fgraph_); fgraph_ = nullptr; }
    }
    if (!fgraph_ && direct_val_ != d_val) {
        // the first factorization from these values is launched directly: a
        // graph pays for its capture only when the plan factors again
        launch_factor(d_val, st);
        direct_val_ = d_val;
        direct = true;
    } else if (!fgraph_) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return SPEIGS_ERR_INTERNAL;
        launch_factor(d_val, st);
        if (cudaStreamEndCapture(st, &g) != cudaSuccess || !g) {
            cudaGetLastError();
            return SPEIGS_ERR_INTERNAL;
        }
        cudaError_t e = cudaGraphInstantiate(&fgraph_, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { cudaGetLastError(); fgraph_ = nullptr; return SPEIGS_ERR_INTERNAL; }
        fgraph_val_ = d_val;
    }
    if (!direct && cudaGraphLaunch(fgraph_, st) != cudaSuccess) {
        cudaGetLastError();
        return SPEIGS_ERR_INTERNAL;
    }
    long long nk = 0;
    for (const MfLaunch &L : launches_) nk += L.count > 0;
    note_launch(nk);
    int h_status = 0;
    cudaMemcpyAsync(&h_status, d_status_, sizeof(int), cudaMemcpyDeviceToHost, st);
    note_d2h(sizeof(int));
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return SPEIGS_ERR_INTERNAL;
    return h_status ? 1 : 0;
}

template <> void MultifrontalPlanT<Real>::solve(const double *b, double *x, cudaStream_t st,
                                                const int *skip) {
    SolveArgs a;
    a.meta = (const SNode *)d_meta_;
    a.tasks = (const STask *)d_stask_;
    a.ntasks = ntasks_;
    a.wtasks = a.tasks + ntasks_;
    a.nfw = nfw_;
    a.nbw = nbw_;
    a.ns = ns_;
    a.bundle = d_bundle_;
    a.perm = d_perm_;
    a.rows = d_rows_;
    a.cptr = d_cptr_;
    a.cidx = d_cidx_;
    a.G = d_G_;
    a.u = d_u_;
    a.yf = d_yf_;
    a.x = d_x_;
    a.fc_base = d_chunks_;
    a.fc_n = d_chunks_ + nfc_;
    a.bc_base = d_chunks_ + 2 * nfc_;
    a.bc_n = d_chunks_ + 2 * nfc_ + nbc_;
    a.fpart = d_fpart_;
    a.bpart = d_bpart_;
    a.fcnt = d_cnt_;
    a.bcnt = d_cnt_ + nfc_;
    a.sync = d_sync_;
    a.b = b;
    a.out = x;
    a.skip = skip;
    // queue, dependency counters and flags start at zero; the error word at
    // the end keeps its value so a failed solve stays visible until read
    cudaMemsetAsync(d_sync_, 0, sizeof(int) * (sync_ints_ - 1), st);
    mf_solve_sf<<<solve_grid_, kSThreads, solve_smem_, st>>>(a);
    note_launch();
}

namespace {
template <int NR>
void launch_bsolve(const BSolveArgs &a, int grid, size_t smem, cudaStream_t st) {
    mf_bsolve<NR><<<grid, kSThreads, smem, st>>>(a);
    note_launch();
}

template <int NR>
int bsolve_config(int *grid, size_t *smem) {
    *smem = bsolve_smem_bytes<NR>();
    if (cudaFuncSetAttribute(mf_bsolve<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)*smem) != cudaSuccess) {
        cudaGetLastError();
        return SPEIGS_ERR_INTERNAL;
    }
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mf_bsolve<NR>, kSThreads, *smem);
    if (per_sm <= 0 || nsm <= 0) return SPEIGS_ERR_INTERNAL;
    *grid = nsm * std::min(per_sm, 4);
    return 0;
}
}  // namespace

template <> int MultifrontalPlanT<Real>::solve_block(const double *B, int64_t ldb, double *X,
                                                     int64_t ldx, int nr, cudaStream_t st,
                                                     const int *skip, bool accumulate) {
    if (nr < 1 || nr > 32 || !d_meta_) return SPEIGS_ERR_ARG;
    const int w = (nr + 7) & ~7;          // 8, 16, 24 or 32 columns per row
    const int q = w / 8 - 1;
    if (w > bw_) {
        // (re)allocate the block buffers for rows of w doubles
        void *old[] = {d_byf_, d_bx_, d_bu_, d_bfp_, d_bbp_};
        for (void *p : old)
            if (p) cudaFreeAsync(p, st);
        d_byf_ = d_bx_ = d_bu_ = d_bfp_ = d_bbp_ = nullptr;
        bw_ = 0;
        int rc = 0;
        rc = rc ? rc : dmalloc(&d_byf_, (size_t)n_ * w, st);
        rc = rc ? rc : dmalloc(&d_bx_, (size_t)n_ * w, st);
        rc = rc ? rc : dmalloc(&d_bu_, (size_t)std::max<int64_t>(u_total_, 1) * w, st);
        rc = rc ? rc : dmalloc(&d_bfp_, (size_t)std::max(fslots_, 1) * kST * w, st);
        rc = rc ? rc : dmalloc(&d_bbp_, (size_t)std::max(bslots_, 1) * kST * w, st);
        if (rc) return rc;
        bw_ = w;
    }
    if (!bgrid_[q]) {
        const int rc = w == 8    ? bsolve_config<8>(&bgrid_[q], &bsmem_[q])
                       : w == 16 ? bsolve_config<16>(&bgrid_[q], &bsmem_[q])
                       : w == 24 ? bsolve_config<24>(&bgrid_[q], &bsmem_[q])
                                 : bsolve_config<32>(&bgrid_[q], &bsmem_[q]);
        if (rc) {
            bgrid_[q] = 0;
            return rc;
        }
    }
    BSolveArgs a;
    a.meta = (const SNode *)d_meta_;
    a.tasks = (const STask *)d_stask_;
    a.ntasks = ntasks_;
    a.wtasks = a.tasks + ntasks_;
    a.nfw = nfw_;
    a.nbw = nbw_;
    a.ns = ns_;
    a.bundle = d_bundle_;
    a.perm = d_perm_;
    a.rows = d_rows_;
    a.cptr = d_cptr_;
    a.cidx = d_cidx_;
    a.G = d_G_;
    a.u = d_bu_;
    a.yf = d_byf_;
    a.x = d_bx_;
    a.fc_base = d_chunks_;
    a.fc_n = d_chunks_ + nfc_;
    a.bc_base = d_chunks_ + 2 * nfc_;
    a.bc_n = d_chunks_ + 2 * nfc_ + nbc_;
    a.fpart = d_bfp_;
    a.bpart = d_bbp_;
    a.fcnt = d_cnt_;
    a.bcnt = d_cnt_ + nfc_;
    a.sync = d_sync_;
    a.bc = B;
    a.xc = X;
    a.ldb = ldb;
    a.ldx = ldx;
    a.nr = nr;
    a.accumulate = accumulate ? 1 : 0;
    a.skip = skip;
    cudaMemsetAsync(d_sync_, 0, sizeof(int) * (sync_ints_ - 1), st);
    if (w == 8)
        launch_bsolve<8>(a, bgrid_[q], bsmem_[q], st);
    else if (w == 16)
        launch_bsolve<16>(a, bgrid_[q], bsmem_[q], st);
    else if (w == 24)
        launch_bsolve<24>(a, bgrid_[q], bsmem_[q], st);
    else
        launch_bsolve<32>(a, bgrid_[q], bsmem_[q], st);
    return 0;
}

template <> int *MultifrontalPlanT<Real>::error_word() const { return d_sync_ ? d_sync_ + (sync_ints_ - 1) : nullptr; }

}  // namespace spx
