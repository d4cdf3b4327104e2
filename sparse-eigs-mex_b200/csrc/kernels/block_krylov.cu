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

// One row range per block: V^T W over the range into part[block], with the
// chunk's rows of V (m columns) and W (b columns) staged in shared memory.
// Thread t owns the outputs (i, j) with i = t % 64 + 64 s (s < 2) and
// j = (t / 64) * 8 + q (q < 8): a warp reads 32 consecutive V columns of a
// row (conflict-free) and one W entry (a broadcast).
__global__ void __launch_bounds__(kTbThreads) tsb_tn_part_kernel(
        const double *__restrict__ V, int64_t ldv, int n, int m, const double *__restrict__ W,
        int64_t ldw, int b, int rows_per_part, double *__restrict__ part) {
    __shared__ double Vs[kTbRows][kBlockMaxM + 1];
    __shared__ double Ws[kTbRows][kBlockMaxB];
    const int t = threadIdx.x;
    const int i0 = t & 63, jg = t >> 6;
    double acc[2][8];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int q = 0; q < 8; q++) acc[s][q] = 0.0;
    const int rb = blockIdx.x * rows_per_part, re = min(n, rb + rows_per_part);
    for (int r0 = rb; r0 < re; r0 += kTbRows) {
        const int nr = min(kTbRows, re - r0);
        for (int e = t; e < kTbRows * kBlockMaxM; e += kTbThreads) {
            const int rr = e % kTbRows, c = e / kTbRows;
            Vs[rr][c] = (rr < nr && c < m) ? V[(int64_t)(r0 + rr) + (int64_t)c * ldv] : 0.0;
        }
        for (int e = t; e < kTbRows * kBlockMaxB; e += kTbThreads) {
            const int rr = e % kTbRows, c = e / kTbRows;
            Ws[rr][c] = (rr < nr && c < b) ? W[(int64_t)(r0 + rr) + (int64_t)c * ldw] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < kTbRows; rr++) {
            const double v0 = Vs[rr][i0], v1 = Vs[rr][i0 + 64];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const double w = Ws[rr][jg * 8 + q];
                acc[0][q] += v0 * w;
                acc[1][q] += v1 * w;
            }
        }
        __syncthreads();
    }
    double *p = part + (size_t)blockIdx.x * (kBlockMaxM * kBlockMaxB);
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int q = 0; q < 8; q++) p[(i0 + 64 * s) * kBlockMaxB + jg * 8 + q] = acc[s][q];
}

// H (=|+=) the sum of the parts, in part order; one thread per output.
__global__ void tsb_tn_reduce_kernel(int m, int b, int nparts, const double *__restrict__ part,
                                     double *H, int ldh, int mode) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= m * kBlockMaxB) return;
    const int i = o / kBlockMaxB, j = o % kBlockMaxB;
    if (j >= b) return;
    double acc = 0.0;
    for (int q = 0; q < nparts; q++) acc += part[(size_t)q * (kBlockMaxM * kBlockMaxB) + o];
    double *h = H + i + (int64_t)j * ldh;
    *h = mode ? *h + acc : acc;
}

// W[row, 0:b] -= V[row, 0:m] H[0:m, 0:b]; one thread per row, H in shared
// memory (read as broadcasts), the row's b sums in registers.
template <int B>
__global__ void __launch_bounds__(256) tsb_nn_sub_kernel(const double *__restrict__ V, int64_t ldv,
                                                         int n, int m, const double *__restrict__ H,
                                                         int ldh, double *W, int64_t ldw, int b) {
    __shared__ double Hs[kBlockMaxM * B];
    for (int e = threadIdx.x; e < m * B; e += blockDim.x) {
        const int i = e / B, j = e % B;
        Hs[e] = (j < b) ? H[i + (int64_t)j * ldh] : 0.0;
    }
    __syncthreads();
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double acc[B];
#pragma unroll
    for (int j = 0; j < B; j++) acc[j] = 0.0;
    for (int i = 0; i < m; i++) {
        const double v = V[(int64_t)row + (int64_t)i * ldv];
#pragma unroll
        for (int j = 0; j < B; j++) acc[j] += v * Hs[i * B + j];
    }
#pragma unroll
    for (int j = 0; j < B; j++)
        if (j < b) W[(int64_t)row + (int64_t)j * ldw] -= acc[j];
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
    }
}

__global__ void __launch_bounds__(256) tsb_right_mul_kernel(int n, int b, double *W, int64_t ldw,
                                                            const double *__restrict__ Rinv) {
    __shared__ double Rs[kBlockMaxB * kBlockMaxB];
    for (int e = threadIdx.x; e < b * b; e += blockDim.x) Rs[e] = Rinv[e];
    __syncthreads();
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double w[kBlockMaxB];
#pragma unroll
    for (int j = 0; j < kBlockMaxB; j++) w[j] = (j < b) ? W[(int64_t)row + (int64_t)j * ldw] : 0.0;
#pragma unroll
    for (int c = 0; c < kBlockMaxB; c++) {
        if (c >= b) break;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < kBlockMaxB; j++)
            if (j <= c) s += w[j] * Rs[j + c * b];
        W[(int64_t)row + (int64_t)c * ldw] = s;
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
    // fixed-order sums per column: thread c takes column c
    bool ok = true;
    for (int c = threadIdx.x; c < b; c += blockDim.x) {
        double t[3] = {0.0, 0.0, 0.0};
        for (int bk = 0; bk < (int)gridDim.x; bk++)
            for (int q = 0; q < 3; q++)
                t[q] += ((volatile double *)part)[(size_t)bk * (3 * BW) + 3 * c + q];
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
    tsb_tn_part_kernel<<<np, kTbThreads, 0, st>>>(V, ldv, n, m, W, ldw, b, rows, bs.part);
    const int outs = m * kBlockMaxB;
    tsb_tn_reduce_kernel<<<(outs + 255) / 256, 256, 0, st>>>(m, b, np, bs.part, H, ldh, mode);
    note_launch(2);
}

void launch_tsb_nn_sub(const double *V, int64_t ldv, int n, int m, const double *H, int ldh,
                       double *W, int64_t ldw, int b, cudaStream_t st) {
    if (m <= 0 || b <= 0) return;
    const int nb = (n + 255) / 256;
    if (b <= 8) tsb_nn_sub_kernel<8><<<nb, 256, 0, st>>>(V, ldv, n, m, H, ldh, W, ldw, b);
    else if (b <= 16) tsb_nn_sub_kernel<16><<<nb, 256, 0, st>>>(V, ldv, n, m, H, ldh, W, ldw, b);
    else tsb_nn_sub_kernel<32><<<nb, 256, 0, st>>>(V, ldv, n, m, H, ldh, W, ldw, b);
    note_launch();
}

void launch_block_chol(int b, const double *G, int ldg, double *Rinv, double abs_floor,
                       double rel_floor, int *status, cudaStream_t st) {
    block_chol_kernel<<<1, 32, 0, st>>>(b, G, ldg, Rinv, abs_floor, rel_floor, status);
    note_launch();
}

void launch_tsb_right_mul(int n, int b, double *W, int64_t ldw, const double *Rinv,
                          cudaStream_t st) {
    tsb_right_mul_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, b, W, ldw, Rinv);
    note_launch();
}

void launch_block_refine_residual(int n, const int32_t *rowptr, const int32_t *col,
                                  const double *val, double shift, const double *B, int64_t ldb,
                                  const double *Y, int64_t ldy, double *R, int64_t ldr, int b,
                                  double tol, double anorm, int *flag, int *count, double *part,
                                  unsigned *counter, cudaStream_t st) {
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
