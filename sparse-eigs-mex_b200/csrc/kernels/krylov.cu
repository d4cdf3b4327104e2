// Krylov-side kernels: FP64 CSR SpMV, tall-skinny Gram-Schmidt passes with a
// deterministic grid reduction, Ritz vectors and true residuals, the
// xorshift64* start vector with exact jump-ahead, and the one-block Jacobi
// eigensolver for the projected matrix.
//
// These replace the BLAS-1/2 and LAPACK calls of the reference's Lanczos
// (src/speigs_core.c): cholmod_l_sdmult in op_multA (:75-83), dgemv T/N in
// orth_block (:122-132), dnrm2/dscal/ddot (:189-191, :209, :223, :251-257),
// dgemv N for Ritz vectors (:250, :278), dsyev (:236) and rand_vec (:49-54).
#include "krylov.cuh"
#include "../common.cuh"
#include "../counters.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>

namespace spx {

// ------------------------------------------------------------------ SpMV --
// One block per 128 consecutive rows.  When the block's nonzeros fit in
// shared memory the products are formed with fully coalesced vector loads --
// a pair of values (16 bytes) and a pair of column indices (8 bytes) per
// thread and step, after at most one leading entry that puts the pairs on
// their 16-byte boundary -- and each thread then sums its own row from
// shared memory (CSR-stream); otherwise a warp walks each row.
constexpr int kSpmvRows = 128;
constexpr int kSpmvCap = 2048;

__global__ void __launch_bounds__(kSpmvRows)
spmv_kernel(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
            const double *__restrict__ va, const double *__restrict__ x,
            double *__restrict__ y) {
    __shared__ double prod[kSpmvCap];
    const int r0 = blockIdx.x * kSpmvRows;
    const int r1 = min(r0 + kSpmvRows, n);
    const int p0 = rp[r0], p1 = rp[r1];
    const int cnt = p1 - p0;
    if (cnt <= kSpmvCap) {
        // entries [p0, p1): an odd p0 is done alone, then aligned pairs, then
        // an odd last entry alone
        const int head = p0 & 1;
        const int npair = (cnt - head) >> 1;
        if (threadIdx.x == 0 && head && cnt > 0) prod[0] = va[p0] * __ldg(x + ci[p0]);
        const double2 *va2 = reinterpret_cast<const double2 *>(va + p0 + head);
        const int2 *ci2 = reinterpret_cast<const int2 *>(ci + p0 + head);
        for (int t = threadIdx.x; t < npair; t += blockDim.x) {
            const double2 v = va2[t];
            const int2 c = ci2[t];
            prod[head + 2 * t] = v.x * __ldg(x + c.x);
            prod[head + 2 * t + 1] = v.y * __ldg(x + c.y);
        }
        const int last = head + 2 * npair;
        if (threadIdx.x == 0 && last < cnt) prod[last] = va[p0 + last] * __ldg(x + ci[p0 + last]);
        __syncthreads();
        const int r = r0 + threadIdx.x;
        if (r < r1) {
            const int a = rp[r] - p0, b = rp[r + 1] - p0;
            double s = 0.0;
            for (int q = a; q < b; q++) s += prod[q];
            y[r] = s;
        }
    } else {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int r = r0 + wid; r < r1; r += blockDim.x >> 5) {
            double s = 0.0;
            for (int q = rp[r] + lane; q < rp[r + 1]; q += 32) s += va[q] * __ldg(x + ci[q]);
            s = warp_sum(s);
            if (lane == 0) y[r] = s;
        }
    }
}

void launch_spmv(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                 const double *x, double *y, cudaStream_t st) {
    if (n <= 0) return;
    int nb = (n + kSpmvRows - 1) / kSpmvRows;
    spmv_kernel<<<nb, kSpmvRows, 0, st>>>(n, rowptr, col, val, x, y);
    note_launch();
}

// ---------------------------------------------------------- tall-skinny --
constexpr int kTsThreads = 256;
constexpr int kTsRows = 2;       // rows per thread
constexpr int kTsChunk = 8;      // columns reduced per register chunk

static int ts_blocks(int n) {
    int nb = (n + kTsThreads * kTsRows - 1) / (kTsThreads * kTsRows);
    return nb < 1 ? 1 : nb;
}

enum { TS_DOT = 0, TS_UPDATE_DOT = 1, TS_UPDATE_NORM = 2, TS_NORM = 3 };

struct TsParams {
    const double *V;
    int64_t ldv;
    int n, m;
    double *w;
    const double *hin;
    double *out;      // h (m) or nrm2 (1)
    double *hcol;     // optional projected-matrix column
    int hmode;        // 0 none, 1 assign, 2 add
    double *part;
    unsigned *counter;
};

// Final cross-block reduction by the last block to arrive: column c of the
// partials is summed over blocks in a fixed order, so results are
// reproducible run to run.
__device__ void last_block_reduce(double *part, unsigned *counter, int ncols, double *out,
                                  double *hcol, int hmode, double *sh) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(counter, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const int nb = gridDim.x;
    const int segs = max(1, (int)blockDim.x / max(ncols, 1));
    const int per = (nb + segs - 1) / segs;
    // sh: ncols * segs doubles
    for (int t = threadIdx.x; t < ncols * segs; t += blockDim.x) {
        int c = t % ncols, s = t / ncols;
        int b0 = s * per, b1 = min(nb, b0 + per);
        // four independent sums keep four L2 loads in flight per thread
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int b = b0;
        for (; b + 3 < b1; b += 4) {
            a0 += __ldcg(part + (size_t)b * ncols + c);
            a1 += __ldcg(part + (size_t)(b + 1) * ncols + c);
            a2 += __ldcg(part + (size_t)(b + 2) * ncols + c);
            a3 += __ldcg(part + (size_t)(b + 3) * ncols + c);
        }
        for (; b < b1; b++) a0 += __ldcg(part + (size_t)b * ncols + c);
        sh[s * ncols + c] = (a0 + a1) + (a2 + a3);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
        double acc = 0.0;
        for (int s = 0; s < segs; s++) acc += sh[s * ncols + c];
        out[c] = acc;
        if (hmode == 1) hcol[c] = acc;
        else if (hmode == 2) hcol[c] += acc;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// One launch covers every row: a block takes 512-row segments
// blockIdx.x, blockIdx.x + gridDim.x, ... (the grid is capped at a few
// blocks per SM), reduces each segment's column sums eight at a time and
// keeps the block's running sums in shared memory; the last block to
// finish combines the blocks' sums.
template <int MODE>
__global__ void __launch_bounds__(kTsThreads) ts_kernel(TsParams p) {
    extern __shared__ double sh[];
    const int n = p.n, m = p.m;
    const int ncols = (MODE == TS_DOT || MODE == TS_UPDATE_DOT) ? m : 1;
    double *hs = sh;                                  // m coefficients
    double *bacc = hs + ((m + 1) & ~1);               // the block's column sums
    double *red = bacc + ((ncols + 1) & ~1);          // block reduce scratch (64)
    double *fin = red + 64;                           // last-block scratch
    if (MODE == TS_UPDATE_DOT || MODE == TS_UPDATE_NORM)
        for (int c = threadIdx.x; c < m; c += blockDim.x) hs[c] = p.hin[c];
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) bacc[c] = 0.0;
    __syncthreads();
    constexpr int kSeg = kTsThreads * kTsRows;
    for (int64_t seg = blockIdx.x; seg * kSeg < n; seg += gridDim.x) {
        const int64_t base = seg * kSeg + threadIdx.x;
        double wv[kTsRows];
#pragma unroll
        for (int r = 0; r < kTsRows; r++) {
            const int64_t i = base + r * kTsThreads;
            wv[r] = (i < n) ? p.w[i] : 0.0;
        }
        if (MODE == TS_UPDATE_DOT || MODE == TS_UPDATE_NORM) {
            double s[kTsRows];
#pragma unroll
            for (int r = 0; r < kTsRows; r++) s[r] = 0.0;
            for (int c = 0; c < m; c++) {
                const double hc = hs[c];
                const double *vc = p.V + (size_t)c * p.ldv;
#pragma unroll
                for (int r = 0; r < kTsRows; r++) {
                    const int64_t i = base + r * kTsThreads;
                    if (i < n) s[r] += vc[i] * hc;
                }
            }
#pragma unroll
            for (int r = 0; r < kTsRows; r++) {
                const int64_t i = base + r * kTsThreads;
                if (i < n) { wv[r] -= s[r]; p.w[i] = wv[r]; }
            }
        }
        if (MODE == TS_DOT || MODE == TS_UPDATE_DOT) {
            for (int c0 = 0; c0 < m; c0 += kTsChunk) {
                double acc[kTsChunk];
#pragma unroll
                for (int q = 0; q < kTsChunk; q++) acc[q] = 0.0;
#pragma unroll
                for (int q = 0; q < kTsChunk; q++) {
                    if (c0 + q < m) {
                        const double *vc = p.V + (size_t)(c0 + q) * p.ldv;
#pragma unroll
                        for (int r = 0; r < kTsRows; r++) {
                            const int64_t i = base + r * kTsThreads;
                            if (i < n) acc[q] += vc[i] * wv[r];
                        }
                    }
                }
                const double t = block_sum8(acc, red);
                if (threadIdx.x < kTsChunk && c0 + (int)threadIdx.x < m) bacc[c0 + threadIdx.x] += t;
            }
        } else {
            double acc = 0.0;
#pragma unroll
            for (int r = 0; r < kTsRows; r++) acc += wv[r] * wv[r];
            const double t = block_sum(acc, red);
            if (threadIdx.x == 0) bacc[0] += t;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < ncols; c += blockDim.x)
        p.part[(size_t)blockIdx.x * ncols + c] = bacc[c];
    last_block_reduce(p.part, p.counter, ncols, p.out, p.hcol, p.hmode, fin);
}

static size_t ts_smem(int ncols_h, int ncols_red) {
    int segs = std::max(1, kTsThreads / std::max(ncols_red, 1));
    return sizeof(double) * ((size_t)((ncols_h + 1) & ~1) + (size_t)((ncols_red + 1) & ~1) + 64 +
                             (size_t)ncols_red * segs);
}

// blocks of a tall-skinny launch: one per 512-row segment, at most four per SM
constexpr int kTsMaxBlocks = 4 * 148;

template <int MODE>
static void ts_launch(const TsParams &p, int ncols_red, cudaStream_t st) {
    int nb = std::min(ts_blocks(p.n), kTsMaxBlocks);
    size_t smem = ts_smem(p.m, ncols_red);
    ts_kernel<MODE><<<nb, kTsThreads, smem, st>>>(p);
    note_launch();
}

void launch_ts_dot(const double *V, int64_t ldv, int n, int m, const double *w, double *h,
                   double *hcol, int hmode, const ReduceScratch &rs, cudaStream_t st) {
    if (m <= 0) return;
    TsParams p{V, ldv, n, m, const_cast<double *>(w), nullptr, h, hcol, hmode, rs.part, rs.counter};
    ts_launch<TS_DOT>(p, m, st);
}
void launch_ts_update_dot(const double *V, int64_t ldv, int n, int m, double *w,
                          const double *hin, double *h, double *hcol, int hmode,
                          const ReduceScratch &rs, cudaStream_t st) {
    if (m <= 0) return;
    TsParams p{V, ldv, n, m, w, hin, h, hcol, hmode, rs.part, rs.counter};
    ts_launch<TS_UPDATE_DOT>(p, m, st);
}
void launch_ts_update_norm(const double *V, int64_t ldv, int n, int m, double *w,
                           const double *hin, double *nrm2, const ReduceScratch &rs,
                           cudaStream_t st) {
    TsParams p{V, ldv, n, m, w, hin, nrm2, nullptr, 0, rs.part, rs.counter};
    if (m <= 0) ts_launch<TS_NORM>(p, 1, st);
    else ts_launch<TS_UPDATE_NORM>(p, 1, st);
}
void launch_ts_norm(int n, const double *w, double *nrm2, const ReduceScratch &rs,
                    cudaStream_t st) {
    TsParams p{nullptr, 0, n, 0, const_cast<double *>(w), nullptr, nrm2, nullptr, 0, rs.part,
               rs.counter};
    ts_launch<TS_NORM>(p, 1, st);
}

__global__ void scale_invnorm_kernel(int n, const double *src, const double *nrm2, double *dst) {
    const double s = 1.0 / sqrt(nrm2[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[i] * s;
}
void launch_scale_by_invnorm(int n, const double *src, const double *nrm2, double *dst,
                             cudaStream_t st) {
    int nb = std::min(4096, (n + 255) / 256);
    scale_invnorm_kernel<<<std::max(nb, 1), 256, 0, st>>>(n, src, nrm2, dst);
    note_launch();
}

// ------------------------------------------------------ Ritz / residual --
struct RitzParams {
    const double *V;
    int64_t ldv;
    int n, m;
    const double *S;
    int lds;
    const int *idx;
    int idx_off, nvec;
    double *X;
    int64_t ldx;
    double *nrm2;
    double *part;
    unsigned *counter;
};

__global__ void __launch_bounds__(kTsThreads) ritz_kernel(RitzParams p) {
    extern __shared__ double sh[];
    const int m = p.m, nv = p.nvec;
    double *Ss = sh;                                  // m x nv
    double *red = Ss + (((size_t)m * nv + 1) & ~1);
    double *fin = red + 32;
    for (int t = threadIdx.x; t < m * nv; t += blockDim.x) {
        int c = t % m, v = t / m;
        Ss[t] = p.S[(size_t)p.idx[p.idx_off + v] * p.lds + c];
    }
    __syncthreads();
    const int base = blockIdx.x * (kTsThreads * kTsRows) + threadIdx.x;
    for (int v0 = 0; v0 < nv; v0 += kTsChunk) {
        double acc[kTsChunk][kTsRows];
#pragma unroll
        for (int q = 0; q < kTsChunk; q++)
#pragma unroll
            for (int r = 0; r < kTsRows; r++) acc[q][r] = 0.0;
        for (int c = 0; c < m; c++) {
            const double *vc = p.V + (size_t)c * p.ldv;
            double vr[kTsRows];
#pragma unroll
            for (int r = 0; r < kTsRows; r++) {
                int i = base + r * kTsThreads;
                vr[r] = (i < p.n) ? vc[i] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < kTsChunk; q++) {
                if (v0 + q < nv) {
                    const double s = Ss[(size_t)(v0 + q) * m + c];
#pragma unroll
                    for (int r = 0; r < kTsRows; r++) acc[q][r] += vr[r] * s;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kTsChunk; q++) {
            if (v0 + q >= nv) continue;
            double sq = 0.0;
#pragma unroll
            for (int r = 0; r < kTsRows; r++) {
                int i = base + r * kTsThreads;
                if (i < p.n) {
                    p.X[(size_t)(v0 + q) * p.ldx + i] = acc[q][r];
                    sq += acc[q][r] * acc[q][r];
                }
            }
            double t = block_sum(sq, red);
            if (threadIdx.x == 0) p.part[(size_t)blockIdx.x * nv + v0 + q] = t;
        }
    }
    last_block_reduce(p.part, p.counter, nv, p.nrm2, nullptr, 0, fin);
}

void launch_ritz_vectors(const double *V, int64_t ldv, int n, int m, const double *S, int lds,
                         const int *idx, int idx_off, int nvec, double *X, int64_t ldx,
                         double *nrm2, const ReduceScratch &rs, cudaStream_t st) {
    if (nvec <= 0) return;
    // vectors per launch: the m x nv block of S fits the default 48 KB of
    // dynamic shared memory beside the reduction scratch
    const int cap = std::max(1, (6144 - 32 - 2 * kTsThreads) / std::max(1, m));
    for (int v0 = 0; v0 < nvec; v0 += cap) {
        const int nv = std::min(cap, nvec - v0);
        RitzParams p{V, ldv, n, m, S, lds, idx, idx_off + v0, nv, X + (size_t)v0 * ldx, ldx,
                     nrm2 + v0, rs.part, rs.counter};
        int nb = ts_blocks(n);
        int segs = std::max(1, kTsThreads / nv);
        size_t smem = sizeof(double) * ((((size_t)m * nv + 1) & ~1) + 32 + (size_t)nv * segs);
        ritz_kernel<<<nb, kTsThreads, smem, st>>>(p);
        note_launch();
    }
}

__global__ void scale_cols_kernel(int n, int nvec, double *X, int64_t ldx, const double *nrm2) {
    const int v = blockIdx.y;
    const double q = nrm2[v];
    if (!(q > 0.0)) return;
    const double s = 1.0 / sqrt(q);
    double *x = X + (size_t)v * ldx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] *= s;
}
void launch_scale_cols(int n, int nvec, double *X, int64_t ldx, const double *nrm2,
                       cudaStream_t st) {
    if (nvec <= 0) return;
    int nb = std::max(1, std::min(1024, (n + 255) / 256));
    scale_cols_kernel<<<dim3(nb, nvec), 256, 0, st>>>(n, nvec, X, ldx, nrm2);
    note_launch();
}

struct RqParams {
    int n, nvec;
    const double *X;
    int64_t ldx;
    const double *AX;
    int64_t ldax;
    double *lam, *r2;
    int pass;
    double *part;
    unsigned *counter;
};

__global__ void __launch_bounds__(kTsThreads) rq_kernel(RqParams p) {
    extern __shared__ double sh[];
    double *red = sh, *fin = sh + 32;
    const int base = blockIdx.x * (kTsThreads * kTsRows) + threadIdx.x;
    for (int v = 0; v < p.nvec; v++) {
        const double *x = p.X + (size_t)v * p.ldx, *ax = p.AX + (size_t)v * p.ldax;
        const double lam = (p.pass == 1) ? p.lam[v] : 0.0;
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < kTsRows; r++) {
            int i = base + r * kTsThreads;
            if (i < p.n) {
                if (p.pass == 0) acc += x[i] * ax[i];
                else { double d = ax[i] - lam * x[i]; acc += d * d; }
            }
        }
        double t = block_sum(acc, red);
        if (threadIdx.x == 0) p.part[(size_t)blockIdx.x * p.nvec + v] = t;
    }
    last_block_reduce(p.part, p.counter, p.nvec, p.pass == 0 ? p.lam : p.r2, nullptr, 0, fin);
}

void launch_rayleigh_resid(int n, int nvec, const double *X, int64_t ldx, const double *AX,
                           int64_t ldax, double *lam, double *r2, const ReduceScratch &rs,
                           cudaStream_t st) {
    if (nvec <= 0) return;
    int nb = ts_blocks(n);
    int segs = std::max(1, kTsThreads / nvec);
    size_t smem = sizeof(double) * (32 + (size_t)nvec * segs);
    for (int pass = 0; pass < 2; pass++) {
        RqParams p{n, nvec, X, ldx, AX, ldax, lam, r2, pass, rs.part, rs.counter};
        rq_kernel<<<nb, kTsThreads, smem, st>>>(p);
        note_launch();
    }
}

// ------------------------------------------------------- refinement ------
// One block per 128 rows (the SpMV layout above); per-block partial sums of
// ||r||^2, ||y||^2 and ||b||^2 are reduced by the last block to arrive, in a
// fixed order, which then takes the convergence decision.
__global__ void __launch_bounds__(kSpmvRows)
refine_residual_kernel(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                       const double *__restrict__ va, double shift, const double *__restrict__ b,
                       const double *__restrict__ y, double *__restrict__ r, double tol,
                       double anorm, int *flag, int *count, double *part, unsigned *counter) {
    __shared__ double red[32];
    __shared__ double fin[3 * kSpmvRows];
    __shared__ bool am_last;
    if (*(volatile const int *)flag) return;
    const int row = blockIdx.x * kSpmvRows + threadIdx.x;
    double r2 = 0.0, y2 = 0.0, b2 = 0.0;
    if (row < n) {
        double s = 0.0;
        for (int q = rp[row]; q < rp[row + 1]; q++) s += va[q] * __ldg(y + ci[q]);
        const double yi = y[row], bi = b[row];
        const double ri = bi - s - shift * yi;
        r[row] = ri;
        r2 = ri * ri;
        y2 = yi * yi;
        b2 = bi * bi;
    }
    r2 = block_sum(r2, red);
    y2 = block_sum(y2, red);
    b2 = block_sum(b2, red);
    if (threadIdx.x == 0) {
        part[(size_t)blockIdx.x * 3 + 0] = r2;
        part[(size_t)blockIdx.x * 3 + 1] = y2;
        part[(size_t)blockIdx.x * 3 + 2] = b2;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // fixed-order reduction: thread t sums blocks t, t+128, ... per column
    for (int c = 0; c < 3; c++) {
        double acc = 0.0;
        for (int bk = threadIdx.x; bk < (int)gridDim.x; bk += blockDim.x)
            acc += ((volatile double *)part)[(size_t)bk * 3 + c];
        fin[c * kSpmvRows + threadIdx.x] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < 3; c++)
            for (int i = 0; i < (int)blockDim.x; i++) t[c] += fin[c * kSpmvRows + i];
        if (sqrt(t[0]) <= tol * (anorm * sqrt(t[1]) + sqrt(t[2]))) *flag = 1;
        else *count += 1;
        *counter = 0u;
    }
}

void launch_refine_residual(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                            double shift, const double *b, const double *y, double *r,
                            double tol, double anorm, int *flag, int *count,
                            const ReduceScratch &rs, cudaStream_t st) {
    const int nb = (n + kSpmvRows - 1) / kSpmvRows;
    refine_residual_kernel<<<nb, kSpmvRows, 0, st>>>(n, rowptr, col, val, shift, b, y, r, tol,
                                                     anorm, flag, count, rs.part, rs.counter);
    note_launch();
}

__global__ void axpy_unless_kernel(int n, double *y, const double *d, const int *flag) {
    if (*(volatile const int *)flag) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] += d[i];
}
void launch_axpy_unless(int n, double *y, const double *d, const int *flag, cudaStream_t st) {
    const int nb = std::max(1, std::min(4096, (n + 255) / 256));
    axpy_unless_kernel<<<nb, 256, 0, st>>>(n, y, d, flag);
    note_launch();
}

// ------------------------------------------------------------ RNG ------
// xorshift64* (reference src/speigs_core.c:49-54).  The state update is
// linear over GF(2), so the state after s steps is M^s applied to the seed;
// the 64 matrices M^(2^b) are tabulated once on the host.
struct JumpTable {
    uint64_t col[64][64];   // col[b][j] = M^(2^b) e_j
};

static uint64_t xs_step(uint64_t x) {
    x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
    return x;
}
static uint64_t apply_mat(const uint64_t *col, uint64_t x) {
    uint64_t y = 0;
    for (int j = 0; j < 64; j++) if ((x >> j) & 1ull) y ^= col[j];
    return y;
}
static const JumpTable &jump_table() {
    static JumpTable T;
    static std::once_flag once;
    std::call_once(once, [] {
        for (int j = 0; j < 64; j++) T.col[0][j] = xs_step(1ull << j);
        for (int b = 1; b < 64; b++)
            for (int j = 0; j < 64; j++) T.col[b][j] = apply_mat(T.col[b - 1], T.col[b - 1][j]);
    });
    return T;
}

const uint64_t *rng_jump_table() { return &jump_table().col[0][0]; }

uint64_t rng_advance(uint64_t seed, uint64_t steps) {
    const JumpTable &T = jump_table();
    for (int b = 0; b < 64; b++)
        if ((steps >> b) & 1ull) seed = apply_mat(T.col[b], seed);
    return seed;
}

constexpr int kRngChunk = 64;

// memory pool of the device (engine.cu): allocations are cached across calls
cudaMemPool_t device_pool(int dev);

__global__ void rand_vec_kernel(int n, uint64_t seed, const uint64_t *__restrict__ jt,
                                double *v) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t first = (int64_t)g * kRngChunk;
    if (first >= n) return;
    uint64_t s = seed;
    uint64_t steps = (uint64_t)first;
    for (int b = 0; steps; b++, steps >>= 1) {
        if (!(steps & 1ull)) continue;
        const uint64_t *col = jt + (size_t)b * 64;
        uint64_t y = 0;
        for (int j = 0; j < 64; j++) y ^= col[j] & (0ull - ((s >> j) & 1ull));
        s = y;
    }
    const int64_t last = min((int64_t)n, first + kRngChunk);
    for (int64_t i = first; i < last; i++) {
        s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
        const uint64_t out = s * 0x2545F4914F6CDD1DULL;
        v[i] = (double)(out >> 11) / 9007199254740992.0 - 0.5;
    }
}

void launch_rand_vec(int n, uint64_t seed, double *v, cudaStream_t st) {
    // the jump table travels with the launch as a small device copy that is
    // owned by this call (no global device state)
    const JumpTable &T = jump_table();
    // (from the library's pool, which keeps its memory: CUDA's default pool
    // returns freed memory to the driver at every synchronisation, and
    // mapping it again on the next call can take milliseconds)
    uint64_t *dj = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool = device_pool(dev);
    cudaError_t ea = pool ? cudaMallocFromPoolAsync((void **)&dj, sizeof(T.col), pool, st)
                          : cudaMallocAsync((void **)&dj, sizeof(T.col), st);
    if (ea != cudaSuccess) { cudaGetLastError(); return; }
    cudaMemcpyAsync(dj, T.col, sizeof(T.col), cudaMemcpyHostToDevice, st);
    note_h2d(sizeof(T.col));
    int threads = (n + kRngChunk - 1) / kRngChunk;
    int nb = (threads + 127) / 128;
    rand_vec_kernel<<<std::max(nb, 1), 128, 0, st>>>(n, seed, dj, v);
    note_launch();
    cudaFreeAsync(dj, st);
}

// -------------------------------------------------- projected eigenproblem --
// Parallel cyclic Jacobi (round-robin pairing, m/2 rotations per round) on
// the symmetric matrix given by the upper triangle of H, in one block.
// Rotation angles follow Rutishauser's formulas; a pair is skipped when
// |a_pq| <= eps * sqrt(|a_pp| |a_qq|), which keeps small eigenvalues
// relatively accurate.  Finishes with eigenvalues ascending (the order dsyev
// returns) and an index list by |theta| descending, stable among ties.
constexpr int kJacThreads = 256;

__device__ void jacobi_body(int m, const double *__restrict__ H, int ldh, double *theta,
                            double *Sout, int *ord, double *gwork, int *status, int use_smem) {
    extern __shared__ double sm[];
    const int me = (m + 1) & ~1;              // even size (a dummy index when m is odd)
    const int half = me / 2;
    double *A, *V, *cs, *sn;
    int *pos;
    if (use_smem) {
        A = sm; V = A + (size_t)me * me;
        cs = V + (size_t)me * me;
    } else {
        A = gwork; V = gwork + (size_t)me * me;
        cs = sm;
    }
    sn = cs + half;
    pos = (int *)(sn + half);
    int *flags = pos + me;                    // [0]: rotated in this sweep
    for (int t = threadIdx.x; t < me * me; t += blockDim.x) {
        int i = t % me, j = t / me;
        double a = 0.0;
        if (i < m && j < m) a = (i <= j) ? H[i + (size_t)j * ldh] : H[j + (size_t)i * ldh];
        A[t] = a;
        V[t] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    // round-robin pairing: index 0 stays, the others shift by one per round,
    // so in round r position t >= 1 holds 1 + ((t - 1 - r) mod (me - 1));
    // phase 1 of a round stores pair pi as (pos[pi], pos[half + pi]), p < q
    auto slot = [&](int t, int r) {
        if (t == 0) return 0;
        int x = t - 1 - r;             // in (-(me - 1), me - 1)
        if (x < 0) x += me - 1;
        return 1 + x;
    };
    int sweep = 0;
    const int max_sweeps = 60;
    for (; sweep < max_sweeps; sweep++) {
        if (threadIdx.x == 0) flags[0] = 0;
        __syncthreads();
        for (int round = 0; round < me - 1; round++) {
            // 1. rotation parameters for every disjoint pair
            for (int pi = threadIdx.x; pi < half; pi += blockDim.x) {
                int p = slot(pi, round), q = slot(me - 1 - pi, round);
                if (p > q) { int t = p; p = q; q = t; }
                pos[pi] = p;
                pos[half + pi] = q;
                double c = 1.0, s = 0.0;
                if (q < m) {
                    const double apq = A[p + (size_t)q * me];
                    const double app = A[p + (size_t)p * me], aqq = A[q + (size_t)q * me];
                    const double thr = DBL_EPSILON * 0.5 * sqrt(fabs(app)) * sqrt(fabs(aqq));
                    if (fabs(apq) > thr && apq != 0.0) {
                        const double th = (aqq - app) / (2.0 * apq);
                        double t;
                        if (fabs(th) > 1e150) t = 0.5 / th;
                        else t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        flags[0] = 1;
                    }
                }
                cs[pi] = c; sn[pi] = s;
            }
            __syncthreads();
            // 2. A <- J^T A J as 2 x 2 blocks (row pair P, column pair Q; the
            // blocks are disjoint, and each is rotated by columns first, then
            // by rows), and V <- V J
            for (int t = threadIdx.x; t < half * half; t += blockDim.x) {
                const int P = t % half, Q = t / half;
                const double c1 = cs[P], s1 = sn[P], c2 = cs[Q], s2 = sn[Q];
                if (s1 == 0.0 && s2 == 0.0) continue;
                const int p1 = pos[P], q1 = pos[half + P], p2 = pos[Q], q2 = pos[half + Q];
                double *a11 = A + p1 + (size_t)p2 * me, *a12 = A + p1 + (size_t)q2 * me;
                double *a21 = A + q1 + (size_t)p2 * me, *a22 = A + q1 + (size_t)q2 * me;
                const double b11 = c2 * *a11 - s2 * *a12, b12 = s2 * *a11 + c2 * *a12;
                const double b21 = c2 * *a21 - s2 * *a22, b22 = s2 * *a21 + c2 * *a22;
                *a11 = c1 * b11 - s1 * b21;
                *a21 = s1 * b11 + c1 * b21;
                *a12 = c1 * b12 - s1 * b22;
                *a22 = s1 * b12 + c1 * b22;
                if (P == Q && s1 != 0.0) { *a12 = 0.0; *a21 = 0.0; }   // exactly decoupled
            }
            for (int t = threadIdx.x; t < half * me; t += blockDim.x) {
                const int Q = t / me, k = t % me;
                const double c = cs[Q], s = sn[Q];
                if (s == 0.0) continue;
                const int p = pos[Q], q = pos[half + Q];
                const double vkp = V[k + (size_t)p * me], vkq = V[k + (size_t)q * me];
                V[k + (size_t)p * me] = c * vkp - s * vkq;
                V[k + (size_t)q * me] = s * vkp + c * vkq;
            }
            __syncthreads();
        }
        int any = flags[0];
        __syncthreads();
        if (!any) break;
    }
    // sort: ascending theta (stable), then by |theta| descending (stable)
    if (threadIdx.x == 0) {
        for (int i = 0; i < m; i++) pos[i] = i;
        for (int i = 1; i < m; i++) {
            int key = pos[i];
            double kv = A[key + (size_t)key * me];
            int j = i - 1;
            while (j >= 0 && A[pos[j] + (size_t)pos[j] * me] > kv) { pos[j + 1] = pos[j]; j--; }
            pos[j + 1] = key;
        }
        for (int i = 0; i < m; i++) ord[i] = i;
        for (int i = 1; i < m; i++) {
            int key = ord[i];
            double kv = fabs(A[pos[key] + (size_t)pos[key] * me]);
            int j = i - 1;
            while (j >= 0 && fabs(A[pos[ord[j]] + (size_t)pos[ord[j]] * me]) < kv) {
                ord[j + 1] = ord[j]; j--;
            }
            ord[j + 1] = key;
        }
        status[0] = (sweep < max_sweeps) ? sweep + 1 : -sweep;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) theta[i] = A[pos[i] + (size_t)pos[i] * me];
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
        int r = t % m, c = t / m;
        Sout[t] = V[r + (size_t)pos[c] * me];
    }
}

__global__ void __launch_bounds__(kJacThreads)
jacobi_kernel(int m, const double *__restrict__ H, int ldh, double *theta, double *Sout,
              int *ord, double *gwork, int *status, int use_smem) {
    jacobi_body(m, H, ldh, theta, Sout, ord, gwork, status, use_smem);
}

// One problem per block: problem b (of order mvec[b] when mvec is given,
// else m) reads H + b * strideH and writes theta, S (ld its order), ord and
// status at b * m, b * m * m, b * m and b * 2; active[b] == 0 skips it.
__global__ void __launch_bounds__(kJacThreads)
jacobi_batched_kernel(int m, const int *mvec, const double *__restrict__ H, int ldh,
                      int64_t strideH, double *theta, double *Sout, int *ord, int *status,
                      const int *active) {
    const int b = blockIdx.x;
    if (active && !active[b]) return;
    const int mb = mvec ? mvec[b] : m;
    jacobi_body(mb, H + (size_t)b * strideH, ldh, theta + (size_t)b * m,
                Sout + (size_t)b * m * m, ord + (size_t)b * m, nullptr, status + 2 * b, 1);
}

static size_t jac_small_bytes(int m) {
    size_t me = (size_t)((m + 1) & ~1);
    return sizeof(double) * (2 * me * me + me) + sizeof(int) * (me + 2);
}

int syev_small_smem_limit() {
    int m = 2;
    while (jac_small_bytes(m + 2) <= 200 * 1024) m += 2;
    return m;
}

void launch_syev_small(int m, const double *H, int ldh, double *theta, double *S, int *ord,
                       double *work, int *status, cudaStream_t st) {
    if (m <= 0) return;
    int use_smem = (m <= syev_small_smem_limit()) ? 1 : 0;
    size_t me = (size_t)((m + 1) & ~1);
    size_t smem = use_smem ? jac_small_bytes(m) : sizeof(double) * me + sizeof(int) * (me + 2);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    jacobi_kernel<<<1, kJacThreads, smem, st>>>(m, H, ldh, theta, S, ord, work, status, use_smem);
    note_launch();
}

void launch_syev_batched(int nprob, int m, const int *mvec, const double *H, int ldh,
                         int64_t strideH, double *theta, double *S, int *ord, int *status,
                         const int *active, cudaStream_t st) {
    if (nprob <= 0 || m <= 0) return;
    const size_t smem = jac_small_bytes(m);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(jacobi_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    jacobi_batched_kernel<<<nprob, kJacThreads, smem, st>>>(m, mvec, H, ldh, strideH, theta, S,
                                                            ord, status, active);
    note_launch();
}

void launch_syev_small_workspace(int m, const double *H, int ldh, double *theta, double *S,
                                 int *ord, double *work, int *status, cudaStream_t st) {
    if (m <= 0) return;
    const size_t me = (size_t)((m + 1) & ~1);
    const size_t smem = sizeof(double) * me + sizeof(int) * (me + 2);
    jacobi_kernel<<<1, kJacThreads, smem, st>>>(m, H, ldh, theta, S, ord, work, status, 0);
    note_launch();
}

__global__ void axpby_kernel(int64_t n, double a, const double *x, double b, double *y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}
void launch_axpby(int64_t n, double a, const double *x, double b, double *y, cudaStream_t st) {
    if (n <= 0) return;
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256));
    axpby_kernel<<<nb, 256, 0, st>>>(n, a, x, b, y);
    note_launch();
}

// ------------------------------------------------------------- helpers --
__global__ void set_diag_kernel(int ldh, int nd, const double *d, double *H) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ldh * ldh; t += gridDim.x * blockDim.x) {
        int i = t % ldh, j = t / ldh;
        H[t] = (i == j && i < nd) ? d[i] : 0.0;
    }
}
void launch_set_diag(int ldh, int nd, const double *d, double *H, cudaStream_t st) {
    int nb = std::max(1, std::min(256, (ldh * ldh + 255) / 256));
    set_diag_kernel<<<nb, 256, 0, st>>>(ldh, nd, d, H);
    note_launch();
}

__global__ void flag_if_below_kernel(const double *nrm2, double thr, int *flag) {
    if (!(nrm2[0] >= thr)) *flag = 1;
}
void launch_flag_if_below(const double *nrm2, double thr, int *flag, cudaStream_t st) {
    flag_if_below_kernel<<<1, 1, 0, st>>>(nrm2, thr, flag);
    note_launch();
}

__global__ void set_beta_kernel(double *H, int ldh, int r, int c, const double *nrm2, int zero) {
    double b = zero ? 0.0 : sqrt(nrm2[0]);
    H[r + (size_t)c * ldh] = b;
    H[c + (size_t)r * ldh] = b;
}
void launch_set_beta(double *H, int ldh, int r, int c, const double *nrm2, int zero,
                     cudaStream_t st) {
    set_beta_kernel<<<1, 1, 0, st>>>(H, ldh, r, c, nrm2, zero);
    note_launch();
}

__global__ void copy_kernel(int64_t n, const double *src, double *dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}
void launch_copy(int64_t n, const double *src, double *dst, cudaStream_t st) {
    if (n <= 0) return;
    int nb = (int)std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256));
    copy_kernel<<<nb, 256, 0, st>>>(n, src, dst);
    note_launch();
}
__global__ void fill_kernel(int64_t n, double v, double *dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}
void launch_fill(int64_t n, double v, double *dst, cudaStream_t st) {
    if (n <= 0) return;
    int nb = (int)std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256));
    fill_kernel<<<nb, 256, 0, st>>>(n, v, dst);
    note_launch();
}

}  // namespace spx

namespace spx {
Counters &counters() {
    static Counters c;
    return c;
}
}  // namespace spx
