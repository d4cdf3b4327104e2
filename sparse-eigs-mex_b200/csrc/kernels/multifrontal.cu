// Device multifrontal supernodal Cholesky (FP64) and the level-scheduled
// shift-invert solve.  See multifrontal.cuh for the storage scheme.
//
// Factorization of one tree level, with T = 32 tiles over each front
// (pivot tiles first, then the tiles of the rows below the pivots):
//   assemble  F = A(pivot columns) + shift*I + extend-add of the children's
//             update matrices (pulled per tile, children in a fixed order)
//   for kb:   potrf of the diagonal tile kb (+ its inverse into G),
//             trsm of the tiles below it (as a product with that inverse),
//             update of the trailing tiles, update matrix included
//   invert    the off-diagonal tiles of inv(L11), row block by row block
//   wmul      G's lower part = L21 * inv(L11)
// A pivot that is not positive records the failing column in a device status
// word (never a trap); later kernels of the same factorization return early.
#include "multifrontal.cuh"
#include "../common.cuh"
#include "../counters.h"

#include <algorithm>
#include <cstring>
#include <new>

#include "../../../include/speigs.h"

namespace spx {

namespace {

constexpr int T = kTile;
constexpr int kFThreads = 256;

struct Sym {
    const int32_t *sfirst, *rows, *relmap, *child_ptr, *child_list;
    const int64_t *rowptr, *frontptr, *gptr;
};

struct Front {
    int64_t fptr, gptr;
    int r, c, nkb, nt, first;
};

SPX_DEV Front front_of(const Sym &y, int s) {
    Front f;
    f.first = y.sfirst[s];
    f.c = y.sfirst[s + 1] - f.first;
    f.r = (int)(y.rowptr[s + 1] - y.rowptr[s]);
    f.nkb = (f.c + T - 1) / T;
    f.nt = f.nkb + (f.r - f.c + T - 1) / T;
    f.fptr = y.frontptr[s];
    f.gptr = y.gptr[s];
    return f;
}

SPX_DEV void tile_range(const Front &f, int I, int &a, int &b) {
    if (I < f.nkb) { a = I * T; b = min(a + T, f.c); }
    else { a = f.c + (I - f.nkb) * T; b = min(a + T, f.r); }
}

// load an h x w tile of a column-major matrix into S[i][j] (zero padded)
SPX_DEV void load_tile(double (*S)[T + 1], const double *M, int64_t ld, int ra, int h, int ca,
                       int w) {
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        int i = t & (T - 1), j = t >> 5;
        S[i][j] = (i < h && j < w) ? M[(int64_t)(ra + i) + (int64_t)(ca + j) * ld] : 0.0;
    }
}

SPX_DEV int lower_bound_i32(const int32_t *a, int n, int key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------ assemble --
__global__ void __launch_bounds__(kFThreads)
mf_assemble(const int4 *__restrict__ tasks, Sym y, double *__restrict__ F,
            const int32_t *__restrict__ acolptr, const int32_t *__restrict__ atpos,
            const int32_t *__restrict__ asrc, const double *__restrict__ val, double shift,
            const int *status) {
    __shared__ double S[T][T + 1];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z;
    const Front f = front_of(y, s);
    int ra, rb, ca, cb;
    tile_range(f, I, ra, rb);
    tile_range(f, J, ca, cb);
    const int h = rb - ra, w = cb - ca;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) S[t & (T - 1)][t >> 5] = 0.0;
    __syncthreads();
    for (int q = y.child_ptr[s]; q < y.child_ptr[s + 1]; q++) {
        const int ch = y.child_list[q];
        const int rch = (int)(y.rowptr[ch + 1] - y.rowptr[ch]);
        const int cch = y.sfirst[ch + 1] - y.sfirst[ch];
        const int nb = rch - cch;
        const int32_t *rm = y.relmap + y.rowptr[ch] + cch;
        const int ia = lower_bound_i32(rm, nb, ra), ib = lower_bound_i32(rm, nb, rb);
        const int ja = lower_bound_i32(rm, nb, ca), jb = lower_bound_i32(rm, nb, cb);
        const int hi = ib - ia, wj = jb - ja;
        if (hi > 0 && wj > 0) {
            const double *U = F + y.frontptr[ch];
            for (int t = threadIdx.x; t < hi * wj; t += blockDim.x) {
                const int i = ia + t % hi, j = ja + t / hi;
                if (i >= j)
                    S[rm[i] - ra][rm[j] - ca] += U[(int64_t)(cch + i) + (int64_t)(cch + j) * rch];
            }
        }
        __syncthreads();
    }
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
    double *Fs = F + f.fptr;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        const int i = t & (T - 1), j = t >> 5;
        if (i < h && j < w) Fs[(int64_t)(ra + i) + (int64_t)(ca + j) * f.r] = S[i][j];
    }
}

// --------------------------------------------------------------- potrf --
__global__ void __launch_bounds__(kFThreads)
mf_potrf(const int4 *__restrict__ tasks, Sym y, double *__restrict__ F, double *__restrict__ G,
         double pivtol, int *status) {
    __shared__ double L[T][T + 1];
    __shared__ double X[T][T + 1];
    if (*(volatile int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, kb = tk.w;
    const Front f = front_of(y, s);
    int a, b;
    tile_range(f, kb, a, b);
    const int w = b - a;
    double *Fs = F + f.fptr;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        const int i = t & (T - 1), j = t >> 5;
        L[i][j] = (i < w && j < w && j <= i) ? Fs[(int64_t)(a + i) + (int64_t)(a + j) * f.r] : 0.0;
        X[i][j] = 0.0;
    }
    __syncthreads();
    for (int j = 0; j < w; j++) {
        if (threadIdx.x == 0) {
            double d = L[j][j];
            if (!(d > pivtol)) {
                atomicCAS(status, 0, f.first + a + j + 1);
                d = 1.0;
            }
            L[j][j] = sqrt(d);
        }
        __syncthreads();
        const double djj = L[j][j];
        if ((int)threadIdx.x > j && (int)threadIdx.x < w) L[threadIdx.x][j] /= djj;
        __syncthreads();
        const int m = w - j - 1;
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            const int i = j + 1 + t % m, k = j + 1 + t / m;
            if (k <= i) L[i][k] -= L[i][j] * L[k][j];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        const int i = t & (T - 1), j = t >> 5;
        if (i < w && j < w && j <= i) Fs[(int64_t)(a + i) + (int64_t)(a + j) * f.r] = L[i][j];
    }
    // X = inv(L): column j by thread j
    if ((int)threadIdx.x < w) {
        const int j = threadIdx.x;
        X[j][j] = 1.0 / L[j][j];
        for (int i = j + 1; i < w; i++) {
            double acc = 0.0;
            for (int t = j; t < i; t++) acc += L[i][t] * X[t][j];
            X[i][j] = -acc / L[i][i];
        }
    }
    __syncthreads();
    double *Gs = G + f.gptr;
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) {
        const int i = t & (T - 1), j = t >> 5;
        if (i < w && j < w && j <= i) Gs[(int64_t)(a + i) + (int64_t)(a + j) * f.r] = X[i][j];
    }
}

// ---------------------------------------------------------- tile products --
// thread (tx, ty) owns C[tx][ty + 8q], q = 0..3
SPX_DEV void mm_abt(double acc[4], const double (*A)[T + 1], const double (*B)[T + 1], int kw) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int t = 0; t < kw; t++) {
        const double av = A[tx][t];
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q] += av * B[ty + 8 * q][t];
    }
}
SPX_DEV void mm_ab(double acc[4], const double (*A)[T + 1], const double (*B)[T + 1], int kw) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int t = 0; t < kw; t++) {
        const double av = A[tx][t];
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q] += av * B[t][ty + 8 * q];
    }
}

// L_Ik = F_Ik * inv(L_kk)^T
__global__ void __launch_bounds__(kFThreads)
mf_trsm(const int4 *__restrict__ tasks, Sym y, double *__restrict__ F,
        const double *__restrict__ G, const int *status) {
    __shared__ double A[T][T + 1];
    __shared__ double X[T][T + 1];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, kb = tk.w;
    const Front f = front_of(y, s);
    int ra, rb, ka, kbb;
    tile_range(f, I, ra, rb);
    tile_range(f, kb, ka, kbb);
    const int h = rb - ra, w = kbb - ka;
    double *Fs = F + f.fptr;
    load_tile(A, Fs, f.r, ra, h, ka, w);
    load_tile(X, G + f.gptr, f.r, ka, w, ka, w);
    __syncthreads();
    double acc[4] = {0, 0, 0, 0};
    mm_abt(acc, A, X, w);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = ty + 8 * q;
        if (tx < h && j < w) Fs[(int64_t)(ra + tx) + (int64_t)(ka + j) * f.r] = acc[q];
    }
}

// F_IJ -= L_Ik L_Jk^T
__global__ void __launch_bounds__(kFThreads)
mf_update(const int4 *__restrict__ tasks, Sym y, double *__restrict__ F, const int *status) {
    __shared__ double A[T][T + 1];
    __shared__ double B[T][T + 1];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z, kb = tk.w;
    const Front f = front_of(y, s);
    int ra, rb, ca, cb, ka, kbb;
    tile_range(f, I, ra, rb);
    tile_range(f, J, ca, cb);
    tile_range(f, kb, ka, kbb);
    const int h = rb - ra, w = cb - ca, kw = kbb - ka;
    double *Fs = F + f.fptr;
    load_tile(A, Fs, f.r, ra, h, ka, kw);
    load_tile(B, Fs, f.r, ca, w, ka, kw);
    __syncthreads();
    double acc[4] = {0, 0, 0, 0};
    mm_abt(acc, A, B, kw);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = ty + 8 * q;
        if (tx < h && j < w) {
            double *p = Fs + (int64_t)(ra + tx) + (int64_t)(ca + j) * f.r;
            *p -= acc[q];
        }
    }
}

// X_ib,jb = -X_ib,ib * sum_{k=jb}^{ib-1} L_ib,k X_k,jb
__global__ void __launch_bounds__(kFThreads)
mf_invert(const int4 *__restrict__ tasks, Sym y, const double *__restrict__ F,
          double *__restrict__ G, const int *status) {
    __shared__ double A[T][T + 1];
    __shared__ double B[T][T + 1];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, ib = tk.y, jb = tk.z;
    const Front f = front_of(y, s);
    int ra, rb, ca, cb;
    tile_range(f, ib, ra, rb);
    tile_range(f, jb, ca, cb);
    const int h = rb - ra, w = cb - ca;
    const double *Fs = F + f.fptr;
    double *Gs = G + f.gptr;
    double acc[4] = {0, 0, 0, 0};
    for (int k = jb; k < ib; k++) {
        int ka, kbb;
        tile_range(f, k, ka, kbb);
        const int kw = kbb - ka;
        load_tile(A, Fs, f.r, ra, h, ka, kw);
        load_tile(B, Gs, f.r, ka, kw, ca, w);
        __syncthreads();
        mm_ab(acc, A, B, kw);
        __syncthreads();
    }
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) B[tx][ty + 8 * q] = acc[q];
    load_tile(A, Gs, f.r, ra, h, ra, h);   // X_ib,ib
    __syncthreads();
    double out[4] = {0, 0, 0, 0};
    mm_ab(out, A, B, h);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = ty + 8 * q;
        if (tx < h && j < w) Gs[(int64_t)(ra + tx) + (int64_t)(ca + j) * f.r] = -out[q];
    }
}

// W_IJ = sum_{K=J}^{nkb-1} L_IK X_KJ   (I a tile of the rows below the pivots)
__global__ void __launch_bounds__(kFThreads)
mf_wmul(const int4 *__restrict__ tasks, Sym y, const double *__restrict__ F,
        double *__restrict__ G, const int *status) {
    __shared__ double A[T][T + 1];
    __shared__ double B[T][T + 1];
    if (*(volatile const int *)status) return;
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, I = tk.y, J = tk.z;
    const Front f = front_of(y, s);
    int ra, rb, ca, cb;
    tile_range(f, I, ra, rb);
    tile_range(f, J, ca, cb);
    const int h = rb - ra, w = cb - ca;
    const double *Fs = F + f.fptr;
    double *Gs = G + f.gptr;
    double acc[4] = {0, 0, 0, 0};
    for (int k = J; k < f.nkb; k++) {
        int ka, kbb;
        tile_range(f, k, ka, kbb);
        const int kw = kbb - ka;
        load_tile(A, Fs, f.r, ra, h, ka, kw);
        load_tile(B, Gs, f.r, ka, kw, ca, w);
        __syncthreads();
        mm_ab(acc, A, B, kw);
        __syncthreads();
    }
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = ty + 8 * q;
        if (tx < h && j < w) Gs[(int64_t)(ra + tx) + (int64_t)(ca + j) * f.r] = acc[q];
    }
}

// ---------------------------------------------------------------- solve --
constexpr int kFwdRows = 64;     // rows of G per forward block
constexpr int kBwdCols = 8;      // columns of G per backward block (one warp each)
constexpr int kSThreads = 256;

struct SolveArgs {
    Sym y;
    const int32_t *perm;
    const int64_t *uptr;
    const double *G;
    double *u, *yf, *x;
};

// forward: f = b(pivots) + children's update vectors; [x1; r2] = G f(0:c);
// yf(pivots) = x1, u_s = f(c:r) - r2
__global__ void __launch_bounds__(kSThreads)
mf_forward(const int4 *__restrict__ tasks, SolveArgs a, const double *__restrict__ bvec) {
    extern __shared__ double fsh[];
    __shared__ double part[4][kFwdRows];
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, chunk = tk.y;
    const Front f = front_of(a.y, s);
    for (int t = threadIdx.x; t < f.r; t += blockDim.x)
        fsh[t] = (t < f.c) ? bvec[a.perm[f.first + t]] : 0.0;
    __syncthreads();
    for (int q = a.y.child_ptr[s]; q < a.y.child_ptr[s + 1]; q++) {
        const int ch = a.y.child_list[q];
        const int rch = (int)(a.y.rowptr[ch + 1] - a.y.rowptr[ch]);
        const int cch = a.y.sfirst[ch + 1] - a.y.sfirst[ch];
        const int32_t *rm = a.y.relmap + a.y.rowptr[ch] + cch;
        const double *uc = a.u + a.uptr[ch];
        for (int i = threadIdx.x; i < rch - cch; i += blockDim.x) fsh[rm[i]] += uc[i];
        __syncthreads();
    }
    const int ri = threadIdx.x % kFwdRows, g = threadIdx.x / kFwdRows;
    const int i = chunk * kFwdRows + ri;
    const double *Gs = a.G + f.gptr;
    double acc = 0.0;
    if (i < f.r) {
        const int jend = (i < f.c) ? i + 1 : f.c;
        for (int j = g; j < jend; j += 4) acc += Gs[(int64_t)i + (int64_t)j * f.r] * fsh[j];
    }
    part[g][ri] = acc;
    __syncthreads();
    if (g == 0 && i < f.r) {
        const double r = (part[0][ri] + part[1][ri]) + (part[2][ri] + part[3][ri]);
        if (i < f.c) a.yf[f.first + i] = r;
        else a.u[a.uptr[s] + (i - f.c)] = fsh[i] - r;
    }
}

// backward: x1 = G^T [yf(pivots); -x(rows below)]
__global__ void __launch_bounds__(kSThreads)
mf_backward(const int4 *__restrict__ tasks, SolveArgs a, double *__restrict__ out) {
    extern __shared__ double vsh[];
    const int4 tk = tasks[blockIdx.x];
    const int s = tk.x, chunk = tk.y;
    const Front f = front_of(a.y, s);
    const int32_t *rows = a.y.rows + a.y.rowptr[s];
    for (int t = threadIdx.x; t < f.r; t += blockDim.x)
        vsh[t] = (t < f.c) ? a.yf[f.first + t] : -a.x[rows[t]];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int j = chunk * kBwdCols + wid;
    if (j >= f.c) return;
    const double *gc = a.G + f.gptr + (int64_t)j * f.r;
    double acc = 0.0;
    for (int i = j + lane; i < f.r; i += 32) acc += gc[i] * vsh[i];
    acc = warp_sum(acc);
    if (lane == 0) {
        a.x[f.first + j] = acc;
        out[a.perm[f.first + j]] = acc;
    }
}

template <class Tp>
static int dmalloc(Tp **p, size_t cnt, cudaStream_t st) {
    if (cudaMallocAsync((void **)p, (cnt ? cnt : 1) * sizeof(Tp), st) != cudaSuccess) {
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

MultifrontalPlan::~MultifrontalPlan() { release(0); }

void MultifrontalPlan::release(cudaStream_t st) {
    void *ptrs[] = {d_perm_, d_sfirst_, d_rows_, d_relmap_, d_child_ptr_, d_child_list_,
                    d_rowptr_, d_frontptr_, d_gptr_, d_uptr_, d_acolptr_, d_atpos_, d_asrc_,
                    d_tasks_, d_stasks_, d_front_, d_G_, d_u_, d_yf_, d_x_, d_status_};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, st);
    d_perm_ = d_sfirst_ = d_rows_ = d_relmap_ = d_child_ptr_ = d_child_list_ = nullptr;
    d_rowptr_ = d_frontptr_ = d_gptr_ = d_uptr_ = nullptr;
    d_acolptr_ = d_atpos_ = d_asrc_ = nullptr;
    d_tasks_ = d_stasks_ = nullptr;
    d_front_ = d_G_ = d_u_ = d_yf_ = d_x_ = nullptr;
    d_status_ = nullptr;
}

int64_t MultifrontalPlan::solve_bytes() const {
    // G read once forward and once backward (lower triangle of the pivot
    // block plus the rows below), the row lists read twice, and the
    // right-hand side, the intermediate and the result vectors.
    return 2 * (8 * g_total_ + 4 * nrows_total_) + 24 * (int64_t)n_;
}

int MultifrontalPlan::init(const spx_symbolic &S, const int64_t *rowptr, const int32_t *col,
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
            gptr[s + 1] = gptr[s] + r * c;
            uptr[s + 1] = uptr[s] + (r - c);
            gtri += c * (c + 1) / 2 + (r - c) * c;
        }
        g_total_ = gtri;
        u_total_ = uptr[ns];
        // assembly entries: for new column j, the entries of A's column
        // perm[j] with new row index >= j, as (row position in the front,
        // index into the CSR values), sorted by row position
        std::vector<int32_t> acolptr(n + 1, 0);
        std::vector<int32_t> atpos, asrc;
        atpos.reserve((size_t)rowptr[n] / 2 + n);
        asrc.reserve((size_t)rowptr[n] / 2 + n);
        std::vector<int32_t> pos(n, -1);
        std::vector<std::pair<int32_t, int32_t>> tmp;
        for (int32_t s = 0; s < ns; s++) {
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
                for (auto &e : tmp) { atpos.push_back(e.first); asrc.push_back(e.second); }
                acolptr[j + 1] = (int32_t)atpos.size();
            }
            for (int64_t t = r0; t < r1; t++) pos[S.rows[t]] = -1;
        }
        // tile task lists, level by level
        std::vector<int4> tasks;
        launches_.clear();
        auto emit = [&](int kind, size_t before) {
            if (tasks.size() > before)
                launches_.push_back({kind, (int64_t)before, (int64_t)(tasks.size() - before)});
        };
        std::vector<int4> stasks;
        fwd_.clear();
        bwd_.clear();
        for (int l = 0; l < S.nlevels; l++) {
            const int32_t q0 = S.level_ptr[l], q1 = S.level_ptr[l + 1];
            int nkbmax = 0;
            size_t b = tasks.size();
            for (int32_t q = q0; q < q1; q++) {
                const int s = S.level_sup[q];
                const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                const int c = S.sfirst[s + 1] - S.sfirst[s];
                const int nkb = (c + T - 1) / T, nt = nkb + (r - c + T - 1) / T;
                nkbmax = std::max(nkbmax, nkb);
                for (int I = 0; I < nt; I++)
                    for (int J = 0; J <= I; J++) tasks.push_back(make_int4(s, I, J, 0));
            }
            emit(MF_ASSEMBLE, b);
            for (int kb = 0; kb < nkbmax; kb++) {
                size_t b0 = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    const int c = S.sfirst[s + 1] - S.sfirst[s];
                    if ((c + T - 1) / T > kb) tasks.push_back(make_int4(s, kb, kb, kb));
                }
                emit(MF_POTRF, b0);
                size_t b1 = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                    const int c = S.sfirst[s + 1] - S.sfirst[s];
                    const int nkb = (c + T - 1) / T, nt = nkb + (r - c + T - 1) / T;
                    if (nkb <= kb) continue;
                    for (int I = kb + 1; I < nt; I++) tasks.push_back(make_int4(s, I, kb, kb));
                }
                emit(MF_TRSM, b1);
                size_t b2 = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                    const int c = S.sfirst[s + 1] - S.sfirst[s];
                    const int nkb = (c + T - 1) / T, nt = nkb + (r - c + T - 1) / T;
                    if (nkb <= kb) continue;
                    for (int I = kb + 1; I < nt; I++)
                        for (int J = kb + 1; J <= I; J++) tasks.push_back(make_int4(s, I, J, kb));
                }
                emit(MF_UPDATE, b2);
            }
            for (int ib = 1; ib < nkbmax; ib++) {
                size_t b0 = tasks.size();
                for (int32_t q = q0; q < q1; q++) {
                    const int s = S.level_sup[q];
                    const int c = S.sfirst[s + 1] - S.sfirst[s];
                    if ((c + T - 1) / T <= ib) continue;
                    for (int jb = 0; jb < ib; jb++) tasks.push_back(make_int4(s, ib, jb, 0));
                }
                emit(MF_INVERT, b0);
            }
            size_t bw = tasks.size();
            for (int32_t q = q0; q < q1; q++) {
                const int s = S.level_sup[q];
                const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                const int c = S.sfirst[s + 1] - S.sfirst[s];
                const int nkb = (c + T - 1) / T, nt = nkb + (r - c + T - 1) / T;
                for (int I = nkb; I < nt; I++)
                    for (int J = 0; J < nkb; J++) tasks.push_back(make_int4(s, I, J, 0));
            }
            emit(MF_WMUL, bw);
            // solve tasks
            size_t f0 = stasks.size();
            for (int32_t q = q0; q < q1; q++) {
                const int s = S.level_sup[q];
                const int r = (int)(S.rowptr[s + 1] - S.rowptr[s]);
                for (int ch = 0; ch * kFwdRows < r; ch++) stasks.push_back(make_int4(s, ch, 0, 0));
            }
            fwd_.push_back({(int64_t)f0, (int64_t)(stasks.size() - f0)});
        }
        for (int l = S.nlevels - 1; l >= 0; l--) {
            size_t b0 = stasks.size();
            for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s = S.level_sup[q];
                const int c = S.sfirst[s + 1] - S.sfirst[s];
                for (int ch = 0; ch * kBwdCols < c; ch++) stasks.push_back(make_int4(s, ch, 0, 0));
            }
            bwd_.push_back({(int64_t)b0, (int64_t)(stasks.size() - b0)});
        }
        int rc = 0;
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
        rc = rc ? rc : dupload(&d_stasks_, stasks.data(), stasks.size(), st);
        rc = rc ? rc : dmalloc(&d_G_, (size_t)gptr[ns], st);
        rc = rc ? rc : dmalloc(&d_u_, (size_t)u_total_, st);
        rc = rc ? rc : dmalloc(&d_yf_, (size_t)n, st);
        rc = rc ? rc : dmalloc(&d_x_, (size_t)n, st);
        rc = rc ? rc : dmalloc(&d_status_, 1, st);
        if (rc) return rc;
        // everything uploaded above comes from host vectors that die here
        if (cudaStreamSynchronize(st) != cudaSuccess) return SPEIGS_ERR_INTERNAL;
        const size_t need = (size_t)max_rows_ * sizeof(double);
        if (need > 48 * 1024) {
            if (need > 227 * 1024) return SPEIGS_ERR_MEM;
            cudaFuncSetAttribute(mf_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
            cudaFuncSetAttribute(mf_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
        }
    } catch (const std::bad_alloc &) {
        return SPEIGS_ERR_MEM;
    }
    return 0;
}

int MultifrontalPlan::factorize(const double *d_val, double shift, double pivtol,
                                cudaStream_t st) {
    if (!d_front_) {
        if (dmalloc(&d_front_, (size_t)front_total_, st)) return SPEIGS_ERR_MEM;
    }
    Sym y{d_sfirst_, d_rows_, d_relmap_, d_child_ptr_, d_child_list_, d_rowptr_, d_frontptr_, d_gptr_};
    // (G's strictly upper pivot part is never written or read)
    cudaMemsetAsync(d_status_, 0, sizeof(int), st);
    for (const MfLaunch &L : launches_) {
        const int4 *tk = d_tasks_ + L.off;
        const unsigned nb = (unsigned)L.count;
        switch (L.kind) {
            case MF_ASSEMBLE:
                mf_assemble<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_acolptr_, d_atpos_,
                                                      d_asrc_, d_val, shift, d_status_);
                note_launch();
                break;
            case MF_POTRF:
                mf_potrf<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_G_, pivtol, d_status_);
                note_launch();
                break;
            case MF_TRSM:
                mf_trsm<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_G_, d_status_);
                note_launch();
                break;
            case MF_UPDATE:
                mf_update<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_status_);
                note_launch();
                break;
            case MF_INVERT:
                mf_invert<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_G_, d_status_);
                note_launch();
                break;
            case MF_WMUL:
                mf_wmul<<<nb, kFThreads, 0, st>>>(tk, y, d_front_, d_G_, d_status_);
                note_launch();
                break;
        }
    }
    int h_status = 0;
    cudaMemcpyAsync(&h_status, d_status_, sizeof(int), cudaMemcpyDeviceToHost, st);
    note_d2h(sizeof(int));
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return SPEIGS_ERR_INTERNAL;
    return h_status ? 1 : 0;
}

void MultifrontalPlan::solve(const double *b, double *x, cudaStream_t st) {
    Sym y{d_sfirst_, d_rows_, d_relmap_, d_child_ptr_, d_child_list_, d_rowptr_, d_frontptr_, d_gptr_};
    SolveArgs a{y, d_perm_, d_uptr_, d_G_, d_u_, d_yf_, d_x_};
    const size_t smem = (size_t)max_rows_ * sizeof(double);
    for (const MfSolveLaunch &L : fwd_)
        if (L.count)
            mf_forward<<<(unsigned)L.count, kSThreads, smem, st>>>(d_stasks_ + L.off, a, b);
            note_launch();
    for (const MfSolveLaunch &L : bwd_)
        if (L.count)
            mf_backward<<<(unsigned)L.count, kSThreads, smem, st>>>(d_stasks_ + L.off, a, x);
            note_launch();
}

}  // namespace spx
