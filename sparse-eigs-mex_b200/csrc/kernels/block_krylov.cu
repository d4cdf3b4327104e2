// Block Krylov kernels (block_krylov.cuh): the tall-skinny products, the
// Cholesky QR and the block refinement residual of the block thick-restart
// Lanczos.  All of them are HBM-bound passes over the basis V (n x m) and
// the block W (n x b); the small dense parts (b x b Cholesky and inverse)
// run in one warp.
#include "block_krylov.cuh"
#include "../common.cuh"
#include "../counters.h"

#include <algorithm>

namespace spx {

namespace {

constexpr int kTbThreads = 256;
constexpr int kTbRows = 32;            // rows per staged chunk
constexpr int kVS = kTbRows + 4;       // padded stride of staged columns / rows (36 doubles)

// m8n8k4 FP64 tensor-core product: lane = 4 gq + tq holds A[gq][tq],
// B[tq][gq] and D[gq][2 tq .. 2 tq + 1]
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}

// One row range per block: V^T W over the range into part[block] on the
// tensor cores.  A 32-row chunk of V's m columns and W's b columns is staged
// column by column (stride kVS, so the fragment reads of a half warp fall in
// distinct banks); warp w owns the 8-row output tiles w and w + 8 of V^T W
// and all of its 8-column tiles.
__device__ __forceinline__ void cp_async8z(double *dst, const double *src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(src),
                 "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(kTbThreads) tsb_tn_part_kernel(
        const double *__restrict__ V, int64_t ldv, int n, int m, const double *__restrict__ W,
        int64_t ldw, int b, int rows_per_part, double *__restrict__ part) {
    // two chunk buffers of (m + b) staged columns: the copies of chunk i+1
    // (cp.async, 8 bytes each, zero-filled past the range) are in flight
    // while chunk i is multiplied
    extern __shared__ double dsm[];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5, gq = lane >> 2, tq = lane & 3;
    const int nmt = (m + 7) >> 3, nnt = (b + 7) >> 3, ncol = m + b;
    double acc[2][4][2];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[s][q][0] = acc[s][q][1] = 0.0;
    const int rb = blockIdx.x * rows_per_part, re = min(n, rb + rows_per_part);
    auto stage = [&](double *Cs, int r0) {
        const int nr = min(kTbRows, re - r0);
        for (int e = t; e < ncol * kTbRows; e += kTbThreads) {
            const int c = e >> 5, rr = e & 31;
            const double *src = (c < m ? V + (int64_t)c * ldv : W + (int64_t)(c - m) * ldw) + r0;
            cp_async8z(Cs + c * kVS + rr, src + (rr < nr ? rr : 0), rr < nr);
        }
        cp_async_commit();
    };
    if (rb < re) stage(dsm, rb);
    int buf = 0;
    for (int r0 = rb; r0 < re; r0 += kTbRows) {
        const double *Cs = dsm + buf * ncol * kVS;
        if (r0 + kTbRows < re) {
            stage(dsm + (buf ^ 1) * ncol * kVS, r0 + kTbRows);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll 2
        for (int ks = 0; ks < kTbRows / 4; ks++) {
            const int k = ks * 4 + tq;
            double bf[4];
#pragma unroll
            for (int q = 0; q < 4; q++) bf[q] = (q * 8 + gq < b) ? Cs[(m + q * 8 + gq) * kVS + k] : 0.0;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int mt = wid + 8 * s;
                if (mt < nmt) {
                    const double a = (mt * 8 + gq < m) ? Cs[(mt * 8 + gq) * kVS + k] : 0.0;
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (q < nnt) dmma884(acc[s][q], a, bf[q]);
                }
            }
        }
        __syncthreads();
        buf ^= 1;
    }
    double *p = part + (size_t)blockIdx.x * (kBlockMaxM * kBlockMaxB);
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int mt = wid + 8 * s;
        if (mt >= nmt) continue;
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (q < nnt)
#pragma unroll
                for (int e = 0; e < 2; e++)
                    p[(mt * 8 + gq) * kBlockMaxB + q * 8 + 2 * tq + e] = acc[s][q][e];
    }
}

// Fused passes over the staged 32-row chunks of one row range, each
// first updating W and then accumulating a product of the updated chunk
// into part[block] exactly as tsb_tn_part_kernel does:
//   kSubTn:   W -= V H1, then V^T W  (the first Gram-Schmidt pass's update
//             and the second pass's product: one read of V for both);
//   kSubGram: W -= V H1, then W^T W  (the second pass's update and the
//             Gram matrix of the Cholesky QR);
//   kMulGram: W = W H1 (H1 = R^{-1}, b x b), then W^T W (a Cholesky QR
//             step and the Gram matrix of the next one).
// The update uses the fragments and the k order of tsb_rows_kernel and the
// product those of tsb_tn_part_kernel, so the results are bit for bit those
// of the separate kernels.  H1 (K x b, leading dimension ldh1; K = m, or b
// for kMulGram) is staged with rows of b + 4 doubles.
enum { kSubTn = 0, kSubGram = 1, kMulGram = 2 };

template <int MODE>
__global__ void __launch_bounds__(kTbThreads) tsb_fused_part_kernel(
        const double *__restrict__ V, int64_t ldv, int n, int m, const double *__restrict__ H1,
        int ldh1, double *__restrict__ W, int64_t ldw, int b, int rows_per_part,
        double *__restrict__ part) {
    extern __shared__ double dsm[];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5, gq = lane >> 2, tq = lane & 3;
    if (MODE == kMulGram) m = 0;                          // no V: the chunk is W alone
    const int nnt = (b + 7) >> 3, ncol = m + b;
    const int K = MODE == kMulGram ? b : m;               // inner size of the update
    const int nks = (K + 3) >> 2, sbs = nnt * 8 + 4;
    // the product's A side: V (kSubTn) or the updated W
    const int pa = MODE == kSubTn ? 0 : m, pm = MODE == kSubTn ? m : b;
    const int nmt = (pm + 7) >> 3;
    double *Bs = dsm + 2 * ncol * kVS;                   // H1: nks * 4 rows of sbs
    for (int e = t; e < nks * 4 * sbs; e += kTbThreads) {
        const int k = e / sbs, j = e % sbs;
        Bs[e] = (k < K && j < b) ? H1[k + (int64_t)j * ldh1] : 0.0;
    }
    double acc[2][4][2];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[s][q][0] = acc[s][q][1] = 0.0;
    const int rb = blockIdx.x * rows_per_part, re = min(n, rb + rows_per_part);
    auto stage = [&](double *Cs, int r0) {
        const int nr = min(kTbRows, re - r0);
        for (int e = t; e < ncol * kTbRows; e += kTbThreads) {
            const int c = e >> 5, rr = e & 31;
            const double *src = (c < m ? V + (int64_t)c * ldv : W + (int64_t)(c - m) * ldw) + r0;
            cp_async8z(Cs + c * kVS + rr, src + (rr < nr ? rr : 0), rr < nr);
        }
        cp_async_commit();
    };
    if (rb < re) stage(dsm, rb);
    int buf = 0;
    for (int r0 = rb; r0 < re; r0 += kTbRows) {
        double *Cs = dsm + buf * ncol * kVS;
        if (r0 + kTbRows < re) {
            stage(dsm + (buf ^ 1) * ncol * kVS, r0 + kTbRows);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        // the update of W[chunk]: output tile ti = (8-row tile ti % 4,
        // 8-column tile ti / 4), tiles taken by the warps in turn; the A
        // side is staged column k (of V, or of W itself for kMulGram, whose
        // products all finish before any of them is written)
        double dv[2][2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int ti = wid + u * (kTbThreads / 32);
            dv[u][0] = dv[u][1] = 0.0;
            if (ti < 4 * nnt) {
                const int rt = ti & 3, q = ti >> 2;
                for (int ks = 0; ks < nks; ks++) {
                    const int k = ks * 4 + tq;
                    const double av = k < K ? Cs[k * kVS + rt * 8 + gq] : 0.0;
                    dmma884(dv[u], av, Bs[k * sbs + q * 8 + gq]);
                }
            }
        }
        if (MODE == kMulGram) __syncthreads();
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int ti = wid + u * (kTbThreads / 32);
            if (ti >= 4 * nnt) continue;
            const int rt = ti & 3, q = ti >> 2, rr = rt * 8 + gq;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = q * 8 + 2 * tq + e;
                if (j < b) {
                    double *cw = Cs + (m + j) * kVS + rr;
                    const double v = MODE == kMulGram ? dv[u][e] : *cw - dv[u][e];
                    *cw = v;
                    if (r0 + rr < re) W[r0 + rr + (int64_t)j * ldw] = v;
                }
            }
        }
        __syncthreads();
#pragma unroll 2
        for (int ks = 0; ks < kTbRows / 4; ks++) {
            const int k = ks * 4 + tq;
            double bf[4];
#pragma unroll
            for (int q = 0; q < 4; q++) bf[q] = (q * 8 + gq < b) ? Cs[(m + q * 8 + gq) * kVS + k] : 0.0;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int mt = wid + 8 * s;
                if (mt < nmt) {
                    const double a = (mt * 8 + gq < pm) ? Cs[(pa + mt * 8 + gq) * kVS + k] : 0.0;
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (q < nnt) dmma884(acc[s][q], a, bf[q]);
                }
            }
        }
        __syncthreads();
        buf ^= 1;
    }
    double *p = part + (size_t)blockIdx.x * (kBlockMaxM * kBlockMaxB);
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int mt = wid + 8 * s;
        if (mt >= nmt) continue;
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (q < nnt)
#pragma unroll
                for (int e = 0; e < 2; e++)
                    p[(mt * 8 + gq) * kBlockMaxB + q * 8 + 2 * tq + e] = acc[s][q][e];
    }
}

// H (=|+=) the sum of the parts: a block per 32 consecutive outputs, warp s
// adding parts s, s + 8, s + 16, ... of each output (coalesced rows of
// part), then the 8 slice sums added in slice order -- a fixed order, so
// the result repeats bit for bit.
constexpr int kRedSlices = 8;
__global__ void __launch_bounds__(32 * kRedSlices) tsb_tn_reduce_kernel(
        int m, int b, int nparts, const double *__restrict__ part, double *H, int ldh, int mode) {
    __shared__ double sl[kRedSlices][33];
    const int lo = threadIdx.x & 31, sli = threadIdx.x >> 5;
    const int o = blockIdx.x * 32 + lo;
    const bool live = o < m * kBlockMaxB;
    double acc = 0.0;
    if (live) {
#pragma unroll 4
        for (int q = sli; q < nparts; q += kRedSlices)
            acc += part[(size_t)q * (kBlockMaxM * kBlockMaxB) + o];
    }
    sl[sli][lo] = acc;
    __syncthreads();
    if (sli != 0 || !live) return;
    const int i = o / kBlockMaxB, j = o % kBlockMaxB;
    if (j >= b) return;
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < kRedSlices; q++) t += sl[q][lo];
    double *h = H + i + (int64_t)j * ldh;
    *h = mode ? *h + t : t;
}

// out[row, 0:b] = W[row, 0:b] - A[row, 0:K] Bm  (SUB), or A[row, 0:K] Bm,
// on the tensor cores: warp w of a block holds 8 rows, Bm (K x b, leading
// dimension ldb) is staged in shared memory with its rows padded to kVS.
// The product overwrites W; with SUB false A may be W itself, since each
// warp reads all of its rows' entries before it writes any.
template <bool SUB>
__global__ void __launch_bounds__(kTbThreads) tsb_rows_kernel(const double *A, int64_t lda, int n,
                                                              int K, const double *Bm, int ldb,
                                                              double *W, int64_t ldw, int b) {
    __shared__ double Bs[kBlockMaxM][kVS];
    const int nks = (K + 3) >> 2;
    for (int e = threadIdx.x; e < nks * 4 * kVS; e += kTbThreads) {
        const int k = e / kVS, j = e % kVS;
        Bs[k][j] = (k < K && j < b) ? Bm[k + (int64_t)j * ldb] : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
    const int r0 = blockIdx.x * (kTbThreads / 4) + wid * 8;
    if (r0 >= n) return;
    const int row = r0 + gq, nnt = (b + 7) >> 3;
    double acc[4][2];
#pragma unroll
    for (int q = 0; q < 4; q++) acc[q][0] = acc[q][1] = 0.0;
    // eight steps' A entries are loaded before they are used, so eight
    // loads per lane are in flight
    for (int ks0 = 0; ks0 < nks; ks0 += 8) {
        double a[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int k = (ks0 + u) * 4 + tq;
            a[u] = (row < n && k < K) ? A[row + (int64_t)k * lda] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            if (ks0 + u >= nks) break;
            const int k = (ks0 + u) * 4 + tq;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < nnt) dmma884(acc[q], a[u], Bs[k][q * 8 + gq]);
        }
    }
    if (row >= n) return;
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (q < nnt)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = q * 8 + 2 * tq + e;
                if (j < b) {
                    double *o = W + row + (int64_t)j * ldw;
                    *o = SUB ? *o - acc[q][e] : acc[q][e];
                }
            }
}

// Cholesky of the column-scaled Gram matrix in one warp (lane j owns
// column j), then the inverse of the upper factor by columns.
__global__ void block_chol_kernel(int b, const double *G, int ldg, double *Rinv, double abs_floor,
                                  double rel_floor, int *status) {
    __shared__ double R[kBlockMaxB][kBlockMaxB + 1];   // R[i][j], upper
    __shared__ double d[kBlockMaxB];
    const int j = threadIdx.x;
    unsigned dep = 0;
    // column scales: unit diagonal after scaling
    double gjj = (j < b) ? G[j + (int64_t)j * ldg] : 1.0;
    const bool zero = (j < b) && !(gjj > abs_floor * abs_floor);
    d[j] = (j < b && !zero) ? sqrt(gjj) : 1.0;
    __syncwarp();
    for (int i = 0; i < kBlockMaxB; i++)
        R[i][j] = (i < b && j < b && i <= j) ? G[i + (int64_t)j * ldg] / (d[i] * d[j]) : 0.0;
    __syncwarp();
    if (zero) dep |= 1u << j;
    // a zero column is replaced: unit pivot, no coupling
    for (int i = 0; i < kBlockMaxB; i++) {
        const unsigned zi = __ballot_sync(0xffffffffu, zero);
        if ((zi >> i) & 1u) R[i][j] = (i == j) ? 1.0 : 0.0;
        if ((zi >> j) & 1u) R[i][j] = (i == j) ? 1.0 : 0.0;
    }
    __syncwarp();
    // right-looking Cholesky: step k scales row k, then updates the trailing rows
    for (int k = 0; k < b; k++) {
        if (j == k) {
            double p = R[k][k];
            if (!(p > rel_floor)) {            // dependent on the columns before it
                dep |= 1u << k;
                R[k][k] = 1.0;
                for (int q = k + 1; q < b; q++) R[k][q] = 0.0;
            } else {
                R[k][k] = sqrt(p);
            }
        }
        __syncwarp();
        const double rkk = R[k][k];
        if (j > k && j < b) R[k][j] /= rkk;
        __syncwarp();
        if (j > k && j < b)
            for (int i = k + 1; i <= j; i++) R[i][j] -= R[k][i] * R[k][j];
        __syncwarp();
    }
    dep = __reduce_or_sync(0xffffffffu, dep);
    // inverse of the scaled factor, column j by back substitution, then
    // the column scaling undone: Rinv = (R D)^{-1} = D^{-1} inv(R) ... applied
    // as Rinv[i][j] = inv(R)[i][j] / d[i] ... with G = D R^T R D, W D^{-1}
    // inv(R) is orthonormal, i.e. Rinv = D^{-1} inv(R)
    double x[kBlockMaxB];
#pragma unroll
    for (int i = 0; i < kBlockMaxB; i++) x[i] = 0.0;
    if (j < b) {
        x[j] = 1.0 / R[j][j];
        for (int i = j - 1; i >= 0; i--) {
            double s = 0.0;
            for (int q = i + 1; q <= j; q++) s += R[i][q] * x[q];
            x[i] = -s / R[i][i];
        }
        for (int i = 0; i < b; i++) Rinv[i + j * b] = (i <= j) ? x[i] / d[i] : 0.0;
    }
    if (j == 0) {
        status[0] = (int)dep;
        status[1] = dep ? 1 : 0;
        if (dep) status[2] = 1;       // sticky until the caller clears it
    }
}

constexpr int kRefRows = 256;

// One thread per row for all b columns: A's row is read once (an SpMM), the
// row's residuals, solution and right-hand-side entries are squared and
// summed per column, first across each warp (shuffles), then across the
// block's warps in shared memory; the block's per-column sums go to part,
// and the last block to finish tests every column in a fixed order.
template <int BW>
__global__ void __launch_bounds__(kRefRows) block_refine_residual_kernel(
        int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
        const double *__restrict__ va, double shift, const double *__restrict__ B, int64_t ldb,
        const double *__restrict__ Y, int64_t ldy, double *__restrict__ R, int64_t ldr, int b,
        double tol, double anorm, int *flag, int *count, double *part, unsigned *counter) {
    __shared__ double wsum[kRefRows / 32][3 * BW];
    __shared__ bool am_last;
    if (*(volatile const int *)flag) return;
    const int row = blockIdx.x * kRefRows + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double acc[BW];
#pragma unroll
    for (int c = 0; c < BW; c++) acc[c] = 0.0;
    if (row < n) {
        for (int q = rp[row]; q < rp[row + 1]; q++) {
            const double a = va[q];
            const int64_t j = ci[q];
#pragma unroll
            for (int c = 0; c < BW; c++)
                if (c < b) acc[c] += a * __ldg(Y + j + (int64_t)c * ldy);
        }
    }
#pragma unroll
    for (int c = 0; c < BW; c++) {
        double r2 = 0.0, y2 = 0.0, b2 = 0.0;
        if (row < n && c < b) {
            const double yi = Y[(int64_t)row + (int64_t)c * ldy];
            const double bi = B[(int64_t)row + (int64_t)c * ldb];
            const double ri = bi - acc[c] - shift * yi;
            R[(int64_t)row + (int64_t)c * ldr] = ri;
            r2 = ri * ri;
            y2 = yi * yi;
            b2 = bi * bi;
        }
        r2 = warp_sum(r2);
        y2 = warp_sum(y2);
        b2 = warp_sum(b2);
        if (lane == 0) {
            wsum[wid][3 * c + 0] = r2;
            wsum[wid][3 * c + 1] = y2;
            wsum[wid][3 * c + 2] = b2;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * b; e += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kRefRows / 32; w++) t += wsum[w][e];
        part[(size_t)blockIdx.x * (3 * BW) + e] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // fixed-order sums: each of the 3 b sums is split over g threads (thread
    // k of the sum takes blocks k, k + g, ...), and the g partial sums are
    // added in thread order -- the same order in every run
    __shared__ double red[kRefRows];
    const int nv = 3 * b, g = kRefRows / nv;
    {
        const int v = threadIdx.x % nv, k = threadIdx.x / nv;
        double t = 0.0;
        if (k < g) {
#pragma unroll 4
            for (int bk = k; bk < (int)gridDim.x; bk += g)
                t += __ldcg(part + (size_t)bk * (3 * BW) + v);
        }
        red[threadIdx.x] = t;
    }
    __syncthreads();
    bool ok = true;
    if ((int)threadIdx.x < b) {
        const int c = threadIdx.x;
        double t[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < g; k++)
#pragma unroll
            for (int q = 0; q < 3; q++) t[q] += red[k * nv + 3 * c + q];
        if (!(sqrt(t[0]) <= tol * (anorm * sqrt(t[1]) + sqrt(t[2])))) ok = false;
    }
    ok = __syncthreads_and(ok);
    if (threadIdx.x == 0) {
        if (ok) *flag = 1;
        else *count += 1;
        *counter = 0u;
    }
}

__global__ void block_axpy_unless_kernel(int n, int b, double *Y, int64_t ldy, const double *D,
                                         int64_t ldd, const int *flag) {
    if (flag && *(volatile const int *)flag) return;
    const int c = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        Y[(int64_t)i + (int64_t)c * ldy] += D[(int64_t)i + (int64_t)c * ldd];
}

__global__ void block_copy_kernel(int n, int b, const double *src, int64_t lds, double *dst,
                                  int64_t ldd) {
    const int c = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[(int64_t)i + (int64_t)c * ldd] = src[(int64_t)i + (int64_t)c * lds];
}

__global__ void block_set_diag_kernel(int ldh, int mm, int l, const double *theta, const int *ord,
                                      double *H) {
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < mm; i += blockDim.x)
        H[i + (int64_t)j * ldh] = (i == j && j < l) ? theta[ord[j]] : 0.0;
}

__global__ void block_ritz_est_kernel(int nwant, int b, const double *S, int lds, int row0,
                                      const int *ord, const double *G, int ldg, double *est2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nwant) return;
    const double *s = S + (int64_t)ord[t] * lds + row0;
    double acc = 0.0;
    for (int i = 0; i < b; i++) {
        double gi = 0.0;
        for (int j = 0; j < b; j++) gi += G[i + (int64_t)j * ldg] * s[j];
        acc += s[i] * gi;
    }
    est2[t] = acc;
}

}  // namespace

int tsb_parts(int n) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) {
            cudaGetLastError();
            nsm = 148;
        }
    }
    const int by_rows = (n + kTbRows - 1) / kTbRows;
    return std::max(1, std::min(2 * nsm, by_rows));
}

void launch_tsb_tn(const double *V, int64_t ldv, int n, int m, const double *W, int64_t ldw,
                   int b, double *H, int ldh, int mode, const BlockScratch &bs, cudaStream_t st) {
    if (m <= 0 || b <= 0) return;
    const int nparts = std::min(tsb_parts(n), bs.max_parts);
    int rows = (n + nparts - 1) / nparts;
    rows = (rows + kTbRows - 1) / kTbRows * kTbRows;
    const int np = (n + rows - 1) / rows;
    const size_t smem = sizeof(double) * 2 * (size_t)(m + b) * kVS;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tsb_tn_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * 2 * (kBlockMaxM + kBlockMaxB) * kVS));
        attr = true;
    }
    tsb_tn_part_kernel<<<np, kTbThreads, smem, st>>>(V, ldv, n, m, W, ldw, b, rows, bs.part);
    const int outs = m * kBlockMaxB;
    tsb_tn_reduce_kernel<<<(outs + 31) / 32, 32 * kRedSlices, 0, st>>>(m, b, np, bs.part, H, ldh,
                                                                       mode);
    note_launch(2);
}

namespace {
// one fused pass (tsb_fused_part_kernel<MODE>) and the reduction of its
// parts into H2 (pm x b, leading dimension ldh2)
template <int MODE>
void launch_fused(const double *V, int64_t ldv, int n, int m, const double *H1, int ldh1,
                  double *W, int64_t ldw, int b, double *H2, int ldh2, int mode,
                  const BlockScratch &bs, cudaStream_t st) {
    const int nparts = std::min(tsb_parts(n), bs.max_parts);
    int rows = (n + nparts - 1) / nparts;
    rows = (rows + kTbRows - 1) / kTbRows * kTbRows;
    const int np = (n + rows - 1) / rows;
    const int mm = MODE == kMulGram ? 0 : m, K = MODE == kMulGram ? b : m;
    const int nnt = (b + 7) >> 3, nks = (K + 3) >> 2;
    const size_t smem =
        sizeof(double) * (2 * (size_t)(mm + b) * kVS + (size_t)nks * 4 * (nnt * 8 + 4));
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tsb_fused_part_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * (2 * (kBlockMaxM + kBlockMaxB) * kVS +
                                                     kBlockMaxM * (kBlockMaxB + 4))));
        attr = true;
    }
    tsb_fused_part_kernel<MODE><<<np, kTbThreads, smem, st>>>(V, ldv, n, mm, H1, ldh1, W, ldw, b,
                                                               rows, bs.part);
    const int pm = MODE == kSubTn ? m : b;
    const int outs = pm * kBlockMaxB;
    tsb_tn_reduce_kernel<<<(outs + 31) / 32, 32 * kRedSlices, 0, st>>>(pm, b, np, bs.part, H2, ldh2,
                                                                       mode);
    note_launch(2);
}
}  // namespace

void launch_tsb_sub_tn(const double *V, int64_t ldv, int n, int m, const double *H1, int ldh1,
                       double *W, int64_t ldw, int b, double *H2, int ldh2, int mode,
                       const BlockScratch &bs, cudaStream_t st) {
    if (m <= 0 || b <= 0) return;
    launch_fused<kSubTn>(V, ldv, n, m, H1, ldh1, W, ldw, b, H2, ldh2, mode, bs, st);
}

void launch_tsb_sub_gram(const double *V, int64_t ldv, int n, int m, const double *H1, int ldh1,
                         double *W, int64_t ldw, int b, double *G, const BlockScratch &bs,
                         cudaStream_t st) {
    if (m <= 0 || b <= 0) return;
    launch_fused<kSubGram>(V, ldv, n, m, H1, ldh1, W, ldw, b, G, b, 0, bs, st);
}

void launch_tsb_mul_gram(int n, int b, double *W, int64_t ldw, const double *Rinv, double *G,
                         const BlockScratch &bs, cudaStream_t st) {
    if (b <= 0) return;
    launch_fused<kMulGram>(nullptr, 0, n, 0, Rinv, b, W, ldw, b, G, b, 0, bs, st);
}

void launch_tsb_nn_sub(const double *V, int64_t ldv, int n, int m, const double *H, int ldh,
                       double *W, int64_t ldw, int b, cudaStream_t st) {
    if (m <= 0 || b <= 0) return;
    const int rows = kTbThreads / 4;
    tsb_rows_kernel<true><<<(n + rows - 1) / rows, kTbThreads, 0, st>>>(V, ldv, n, m, H, ldh, W,
                                                                        ldw, b);
    note_launch();
}

void launch_block_chol(int b, const double *G, int ldg, double *Rinv, double abs_floor,
                       double rel_floor, int *status, cudaStream_t st) {
    block_chol_kernel<<<1, 32, 0, st>>>(b, G, ldg, Rinv, abs_floor, rel_floor, status);
    note_launch();
}

void launch_tsb_right_mul(int n, int b, double *W, int64_t ldw, const double *Rinv,
                          cudaStream_t st) {
    if (b <= 0) return;
    const int rows = kTbThreads / 4;
    tsb_rows_kernel<false><<<(n + rows - 1) / rows, kTbThreads, 0, st>>>(W, ldw, n, b, Rinv, b, W,
                                                                         ldw, b);
    note_launch();
}

void launch_tsb_right_mul_into(int n, int K, const double *X, int64_t ldx, const double *S,
                               int lds, double *W, int64_t ldw, int b, cudaStream_t st) {
    if (b <= 0 || K <= 0) return;
    const int rows = kTbThreads / 4;
    tsb_rows_kernel<false><<<(n + rows - 1) / rows, kTbThreads, 0, st>>>(X, ldx, n, K, S, lds, W,
                                                                         ldw, b);
    note_launch();
}

void launch_block_refine_residual(int n, const int32_t *rowptr, const int32_t *col,
                                  const double *val, double shift, const double *B, int64_t ldb,
                                  const double *Y, int64_t ldy, double *R, int64_t ldr, int b,
                                  double tol, double anorm, int *flag, int *count, double *part,
                                  unsigned *counter, cudaStream_t st) {
    if (b <= 0) return;
    const int grid = (n + kRefRows - 1) / kRefRows;
#define SPX_REFINE(BW)                                                                        \
    block_refine_residual_kernel<BW><<<grid, kRefRows, 0, st>>>(n, rowptr, col, val, shift, B, \
                                                                ldb, Y, ldy, R, ldr, b, tol,  \
                                                                anorm, flag, count, part,     \
                                                                counter)
    if (b <= 8) SPX_REFINE(8);
    else if (b <= 16) SPX_REFINE(16);
    else SPX_REFINE(32);
#undef SPX_REFINE
    note_launch();
}

void launch_block_axpy_unless(int n, int b, double *Y, int64_t ldy, const double *D,
                              int64_t ldd, const int *flag, cudaStream_t st) {
    dim3 grid(std::max(1, std::min(1024, (n + 255) / 256)), b);
    block_axpy_unless_kernel<<<grid, 256, 0, st>>>(n, b, Y, ldy, D, ldd, flag);
    note_launch();
}

void launch_block_copy(int n, int b, const double *src, int64_t lds, double *dst, int64_t ldd,
                       cudaStream_t st) {
    if (b <= 0) return;
    dim3 grid(std::max(1, std::min(1024, (n + 255) / 256)), b);
    block_copy_kernel<<<grid, 256, 0, st>>>(n, b, src, lds, dst, ldd);
    note_launch();
}

void launch_block_set_diag(int ldh, int mm, int l, const double *theta, const int *ord,
                           double *H, cudaStream_t st) {
    block_set_diag_kernel<<<mm, 128, 0, st>>>(ldh, mm, l, theta, ord, H);
    note_launch();
}

void launch_block_ritz_est(int nwant, int b, const double *S, int lds, int row0, const int *ord,
                           const double *G, int ldg, double *est2, cudaStream_t st) {
    block_ritz_est_kernel<<<(nwant + 63) / 64, 64, 0, st>>>(nwant, b, S, lds, row0, ord, G, ldg,
                                                            est2);
    note_launch();
}

}  // namespace spx
