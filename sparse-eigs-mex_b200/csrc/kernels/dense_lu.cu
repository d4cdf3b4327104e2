// Gauss-Jordan inverse with partial pivoting (dense_lu.cuh).
//
// In-place elimination: at step k the pivot row p (largest |M[i][k]|,
// i >= k, the smallest such i on ties) is swapped into row k, then every
// entry is updated from the pivot row and column copied aside by the same
// step:
//   M[k][k] = 1/piv,  M[k][j] = M[k][j]/piv,  M[i][k] = -M[i][k]/piv,
//   M[i][j] -= M[i][k] M[k][j] / piv        (i != k, j != k).
// After the n steps M is (P A)^{-1}; undoing the row interchanges as column
// interchanges in reverse order gives A^{-1}.  Each step is two launches: a
// one-block pivot search and row swap, and a grid-wide rank-one update, so
// the route is HBM-bound: 16 n^3 bytes in all.
#include "dense_lu.cuh"
#include "../common.cuh"
#include "../counters.h"

#include <algorithm>
#include <cfloat>
#include <vector>

namespace spx {

namespace {

constexpr int kPivThreads = 1024;

__global__ void densify_cm_kernel(int n, const int32_t *rp, const int32_t *ci, const double *va,
                                  double *M) {
    for (int r = blockIdx.x; r < n; r += gridDim.x)
        for (int q = rp[r] + threadIdx.x; q < rp[r + 1]; q += blockDim.x)
            M[(int64_t)r + (int64_t)ci[q] * n] = va[q];
}

// pivot search over column k, row swap, copies of the pivot row and column
__global__ void __launch_bounds__(kPivThreads) gj_pivot_kernel(int n, int k, double *M,
                                                               double *rowbuf, double *colbuf,
                                                               int *ipiv, int *flags, double tiny) {
    __shared__ double sv[kPivThreads];
    __shared__ int si[kPivThreads];
    const int t = threadIdx.x;
    const double *colk = M + (int64_t)k * n;
    double best = -1.0;
    int bi = n;
    for (int i = k + t; i < n; i += blockDim.x) {
        const double a = fabs(colk[i]);
        if (a > best) { best = a; bi = i; }   // first maximum in this thread's rows
    }
    sv[t] = best;
    si[t] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            const double a = sv[t + s];
            const int ia = si[t + s];
            if (a > sv[t] || (a == sv[t] && ia < si[t])) { sv[t] = a; si[t] = ia; }
        }
        __syncthreads();
    }
    const int p = si[0];
    if (t == 0) ipiv[k] = p;
    if (p != k)
        for (int j = t; j < n; j += blockDim.x) {
            const double a = M[(int64_t)k + (int64_t)j * n], b = M[(int64_t)p + (int64_t)j * n];
            M[(int64_t)k + (int64_t)j * n] = b;
            M[(int64_t)p + (int64_t)j * n] = a;
        }
    __syncthreads();
    for (int j = t; j < n; j += blockDim.x) {
        rowbuf[j] = M[(int64_t)k + (int64_t)j * n];
        colbuf[j] = colk[j];
    }
    __syncthreads();
    if (t == 0 && M[(int64_t)k + (int64_t)k * n] == 0.0) {
        // singular to working precision: a tiny pivot keeps the inverse finite
        rowbuf[k] = tiny;
        colbuf[k] = tiny;
        flags[0] = 1;
    }
}

__global__ void gj_update_kernel(int n, int k, double *M, const double *__restrict__ rowbuf,
                                 const double *__restrict__ colbuf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const double piv = colbuf[k];
    const double inv = 1.0 / piv;
    double *m = M + (int64_t)i + (int64_t)j * n;
    if (i == k && j == k) *m = inv;
    else if (i == k) *m = rowbuf[j] * inv;
    else if (j == k) *m = -colbuf[i] * inv;
    else *m -= colbuf[i] * (rowbuf[j] * inv);
}

__global__ void swap_cols_kernel(int n, int a, int b, double *M) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = M[(int64_t)i + (int64_t)a * n];
        M[(int64_t)i + (int64_t)a * n] = M[(int64_t)i + (int64_t)b * n];
        M[(int64_t)i + (int64_t)b * n] = x;
    }
}

// one warp per output: y[i] = column i of M . x
__global__ void dense_apply_kernel(int n, const double *__restrict__ M, const double *__restrict__ x,
                                   double *y) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    const double *c = M + (int64_t)w * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += c[j] * x[j];
    acc = warp_sum(acc);
    if (lane == 0) y[w] = acc;
}

}  // namespace

void launch_dense_inverse(int n, const int32_t *rowptr, const int32_t *col, const double *val,
                          double anorm, double *M, double *rowbuf, double *colbuf, int *ipiv,
                          int *flags, cudaStream_t st) {
    cudaMemsetAsync(M, 0, sizeof(double) * (size_t)n * n, st);
    cudaMemsetAsync(flags, 0, sizeof(int) * 2, st);
    densify_cm_kernel<<<std::min(n, 4096), 32, 0, st>>>(n, rowptr, col, val, M);
    const double tiny = DBL_EPSILON * (anorm > 0 ? anorm : 1.0);
    const dim3 ug((n + 255) / 256, n);
    for (int k = 0; k < n; k++) {
        gj_pivot_kernel<<<1, kPivThreads, 0, st>>>(n, k, M, rowbuf, colbuf, ipiv, flags, tiny);
        gj_update_kernel<<<ug, 256, 0, st>>>(n, k, M, rowbuf, colbuf);
    }
    // the row interchanges, undone as column interchanges in reverse order
    // (ipiv is read back: the order is data dependent)
    std::vector<int> hp(n);
    cudaMemcpyAsync(hp.data(), ipiv, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    note_d2h((long long)sizeof(int) * n);
    cudaStreamSynchronize(st);
    long long nl = 1 + 2LL * n;
    for (int k = n - 1; k >= 0; k--)
        if (hp[k] != k) {
            swap_cols_kernel<<<std::max(1, std::min(64, (n + 255) / 256)), 256, 0, st>>>(n, k, hp[k],
                                                                                        M);
            nl++;
        }
    note_launch(nl);
}

void launch_dense_apply(int n, const double *M, const double *x, double *y, cudaStream_t st) {
    const int threads = 256;
    const int blocks = (int)(((int64_t)n * 32 + threads - 1) / threads);
    dense_apply_kernel<<<blocks, threads, 0, st>>>(n, M, x, y);
    note_launch();
}

}  // namespace spx
