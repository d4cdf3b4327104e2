// Message-passing network that proposes a start subspace for the Lanczos
// iteration of a finite-volume diffusion operator (the learned warm start).
//
//   h0   = tanh(W0 x + b0)                          x: F node features
//   h_l  = tanh(W_l [h_{l-1}, A h_{l-1}] + b_l)     l = 1..L, A the normalised
//                                                   adjacency of the operator
//   Y    = W_o h_L + b_o                            P outputs per node
//
// Activations are stored in BF16, weights are used in BF16 and kept in FP32
// for the optimiser; every product accumulates in FP32.  Training minimises
// the subspace loss 1 - trace(U^T P_Y U) / k, P_Y the orthogonal projector
// onto span(Y) and U the k eigenvectors the solver computed for the same
// operator; its gradient is dL/dY = -(2/k) (U - Y C) C^T with
// C = (Y^T Y)^{-1} Y^T U.  Adam updates the FP32 weights.
#include "../common.cuh"
#include "../counters.h"
#include "../../../include/speigs_b200.h"

#include <cub/device/device_scan.cuh>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace spx {
const char *set_last_error_text(const char *msg);
cudaMemPool_t device_pool(int dev);
}

namespace {

using bf16 = __nv_bfloat16;
constexpr int kRows = 64;       // nodes per block in the dense layers
constexpr int kThreads = 256;

SPX_DEV float to_f(bf16 v) { return __bfloat162float(v); }
SPX_DEV float to_f(float v) { return v; }
template <class T> SPX_DEV T from_f(float v);
template <> SPX_DEV bf16 from_f<bf16>(float v) { return __float2bfloat16(v); }
template <> SPX_DEV float from_f<float>(float v) { return v; }

// ---- message passing: out = A in (one warp per node, 2 features a lane)
template <class TI, class TO>
__global__ void spmm_kernel(int n, int hid, const int32_t *__restrict__ rp,
                            const int32_t *__restrict__ ci, const float *__restrict__ w,
                            const TI *__restrict__ in, TO *__restrict__ out, int accumulate) {
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    for (int f0 = 0; f0 < hid; f0 += 64) {
        float a0 = 0.f, a1 = 0.f;
        const int f = f0 + 2 * lane;
        for (int q = rp[row]; q < rp[row + 1]; q++) {
            const float wq = w[q];
            const TI *src = in + (size_t)ci[q] * hid;
            if (f < hid) a0 += wq * to_f(src[f]);
            if (f + 1 < hid) a1 += wq * to_f(src[f + 1]);
        }
        TO *dst = out + (size_t)row * hid;
        if (f < hid) dst[f] = from_f<TO>(accumulate ? to_f(dst[f]) + a0 : a0);
        if (f + 1 < hid) dst[f + 1] = from_f<TO>(accumulate ? to_f(dst[f + 1]) + a1 : a1);
    }
}

// ---- dense layer forward: out[i, o] = act(b[o] + sum_k W[o, k] x[i, k]),
// x = [X1[i, 0:K1], X2[i, 0:K2]] (X2 may be absent).  act: 0 identity, 1 tanh.
template <class T1, class TO>
__global__ void __launch_bounds__(kThreads)
dense_fwd_kernel(int n, int K1, const T1 *__restrict__ X1, int K2, const bf16 *__restrict__ X2,
                 int N, const bf16 *__restrict__ W, const float *__restrict__ b, int act,
                 TO *__restrict__ out) {
    extern __shared__ float sm[];
    const int K = K1 + K2;
    float *Xs = sm;                       // kRows x (K + 1)
    float *Ws = Xs + kRows * (K + 1);     // N x (K + 1)
    const int r0 = blockIdx.x * kRows;
    for (int t = threadIdx.x; t < kRows * K; t += blockDim.x) {
        const int r = t / K, k = t % K, i = r0 + r;
        float v = 0.f;
        if (i < n) v = (k < K1) ? to_f(X1[(size_t)i * K1 + k]) : to_f(X2[(size_t)i * K2 + (k - K1)]);
        Xs[r * (K + 1) + k] = v;
    }
    for (int t = threadIdx.x; t < N * K; t += blockDim.x) Ws[(t / K) * (K + 1) + t % K] = to_f(W[t]);
    __syncthreads();
    for (int t = threadIdx.x; t < kRows * N; t += blockDim.x) {
        const int r = t / N, o = t % N, i = r0 + r;
        if (i >= n) continue;
        float acc = b[o];
        const float *xr = Xs + r * (K + 1), *wr = Ws + o * (K + 1);
        for (int k = 0; k < K; k++) acc += xr[k] * wr[k];
        out[(size_t)i * N + o] = from_f<TO>(act ? tanhf(acc) : acc);
    }
}

// ---- dense layer backward.  dZ = dOut * act'(out); dX1/dX2 (FP32; added
// when `accumulate`) = dZ W; dW += dZ^T x; db += column sums of dZ.
template <class T1, class TOut>
__global__ void __launch_bounds__(kThreads)
dense_bwd_kernel(int n, int K1, const T1 *__restrict__ X1, int K2, const bf16 *__restrict__ X2,
                 int N, const bf16 *__restrict__ W, int act, const TOut *__restrict__ out,
                 const float *__restrict__ dout, float *dX1, float *dX2, int accumulate,
                 float *__restrict__ dW, float *__restrict__ db) {
    extern __shared__ float sm[];
    const int K = K1 + K2;
    float *Xs = sm;                        // kRows x (K + 1)
    float *Ws = Xs + kRows * (K + 1);      // N x (K + 1)
    float *Zs = Ws + N * (K + 1);          // kRows x (N + 1)
    const int r0 = blockIdx.x * kRows;
    for (int t = threadIdx.x; t < kRows * K; t += blockDim.x) {
        const int r = t / K, k = t % K, i = r0 + r;
        float v = 0.f;
        if (i < n) v = (k < K1) ? to_f(X1[(size_t)i * K1 + k]) : to_f(X2[(size_t)i * K2 + (k - K1)]);
        Xs[r * (K + 1) + k] = v;
    }
    for (int t = threadIdx.x; t < N * K; t += blockDim.x) Ws[(t / K) * (K + 1) + t % K] = to_f(W[t]);
    for (int t = threadIdx.x; t < kRows * N; t += blockDim.x) {
        const int r = t / N, o = t % N, i = r0 + r;
        float z = 0.f;
        if (i < n) {
            z = dout[(size_t)i * N + o];
            if (act) {
                const float y = to_f(out[(size_t)i * N + o]);
                z *= 1.f - y * y;
            }
        }
        Zs[r * (N + 1) + o] = z;
    }
    __syncthreads();
    // dX = dZ W
    if (dX1 || dX2)
        for (int t = threadIdx.x; t < kRows * K; t += blockDim.x) {
            const int r = t / K, k = t % K, i = r0 + r;
            if (i >= n) continue;
            float acc = 0.f;
            for (int o = 0; o < N; o++) acc += Zs[r * (N + 1) + o] * Ws[o * (K + 1) + k];
            float *dst = (k < K1) ? (dX1 ? dX1 + (size_t)i * K1 + k : nullptr)
                                  : (dX2 ? dX2 + (size_t)i * K2 + (k - K1) : nullptr);
            if (dst) *dst = accumulate ? *dst + acc : acc;
        }
    // dW += dZ^T x, db += sum dZ
    for (int t = threadIdx.x; t < N * (K + 1); t += blockDim.x) {
        const int o = t / (K + 1), k = t % (K + 1);
        float acc = 0.f;
        if (k < K)
            for (int r = 0; r < kRows; r++) acc += Zs[r * (N + 1) + o] * Xs[r * (K + 1) + k];
        else
            for (int r = 0; r < kRows; r++) acc += Zs[r * (N + 1) + o];
        if (acc != 0.f) {
            if (k < K) atomicAdd(dW + (size_t)o * K + k, acc);
            else atomicAdd(db + o, acc);
        }
    }
}

// ---- dense layer forward on the tensor cores (tcgen05, TMEM accumulator)
// out[i, o] = act(b[o] + sum_k W[o, k] x[i, k]) as dense_fwd_kernel, for BF16
// inputs x = [X1[i, 0:K1], X2[i, 0:K2]] (K1, K2 multiples of 8, K = K1 + K2 a
// multiple of 16, at most 128) and N <= 64 outputs.  One block of 4 warps
// takes 128 rows:
//   * the rows (A, 128 x K) and W (B, NP x K, NP = N rounded up to 16, rows
//     >= N zero) are staged in shared memory in the K-major layout without
//     swizzle that tcgen05 descriptors address: 8-row x 16-byte core
//     matrices, the K chunks of one 8-row group 128 bytes apart (leading
//     byte offset), 8-row groups K/8 x 128 bytes apart (stride byte offset);
//   * one thread issues K/16 tcgen05.mma kind::f16 (M = 128, N = NP, K = 16,
//     BF16 operands, FP32 accumulation) into NP columns of TMEM and commits
//     them to an mbarrier;
//   * each warp reads its 32 TMEM lanes -- lane = row -- with tcgen05.ld and
//     applies bias and activation; a thread stores its row in 16-byte pieces.
// The mbarrier wait is bounded: when it runs out, *err is set, the block
// waits (bounded) once more for its MMAs, frees its TMEM and stores nothing.
constexpr int kTcRows = 128;
constexpr int kTcThreads = 128;
constexpr long kTcSpin = 1L << 22;

SPX_DEV uint32_t sh_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading and stride byte
// offsets (16-byte units), descriptor version 1, no swizzle
SPX_DEV uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 D (bits 4-5 = 1), BF16 A and B
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t umma_idesc_bf16(int nn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nn >> 3) << 17) |
           ((uint32_t)(kTcRows >> 4) << 24);
}
SPX_DEV bool tc_bar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
SPX_DEV float tc_act(float v, int act) { return act ? tanhf(v) : v; }

template <class TO>
__global__ void __launch_bounds__(kTcThreads)
dense_fwd_tc_kernel(int n, int K1, const bf16 *__restrict__ X1, int K2, const bf16 *__restrict__ X2,
                    int N, int NP, const bf16 *__restrict__ W, const float *__restrict__ b, int act,
                    TO *__restrict__ out, volatile int *err) {
    extern __shared__ __align__(1024) unsigned char tc_sm[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) unsigned long long s_bar;
    const int K = K1 + K2, KC = K >> 3, KC1 = K1 >> 3;
    const uint32_t sbo = (uint32_t)KC * 128u;
    unsigned char *sA = tc_sm, *sB = tc_sm + (size_t)kTcRows * K * 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = NP <= 32 ? 32u : 64u;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(sh_addr(&s_tmem)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sh_addr(&s_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const int row0 = blockIdx.x * kTcRows;
    // A: 128 rows x KC chunks; consecutive threads take the 8 rows of a core
    // matrix, then the next chunk (512 contiguous bytes a warp)
    for (int idx = threadIdx.x; idx < kTcRows * KC; idx += kTcThreads) {
        const int r0 = idx & 7, c = (idx >> 3) % KC, r1 = (idx >> 3) / KC;
        const int i = row0 + r1 * 8 + r0;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (i < n)
            v = c < KC1 ? *reinterpret_cast<const uint4 *>(X1 + (size_t)i * K1 + c * 8)
                        : *reinterpret_cast<const uint4 *>(X2 + (size_t)i * K2 + (c - KC1) * 8);
        *reinterpret_cast<uint4 *>(sA + r0 * 16 + r1 * sbo + c * 128) = v;
    }
    // B: NP rows of W (rows >= N zero)
    for (int idx = threadIdx.x; idx < NP * KC; idx += kTcThreads) {
        const int r0 = idx & 7, c = (idx >> 3) % KC, r1 = (idx >> 3) / KC;
        const int o = r1 * 8 + r0;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (o < N) v = *reinterpret_cast<const uint4 *>(W + (size_t)o * K + c * 8);
        *reinterpret_cast<uint4 *>(sB + r0 * 16 + r1 * sbo + c * 128) = v;
    }
    // the generic-proxy stores above become visible to the tensor core's reads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t bar = sh_addr(&s_bar);
    if (threadIdx.x == 0) {
        const uint32_t idesc = umma_idesc_bf16(NP);
        const uint32_t a0 = sh_addr(sA), b0 = sh_addr(sB);
        for (int j = 0; j < (K >> 4); j++) {
            const uint64_t da = umma_desc(a0 + 256u * j, 128u, sbo);
            const uint64_t db = umma_desc(b0 + 256u * j, 128u, sbo);
            const uint32_t acc = j > 0 ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}"
                ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(bar) : "memory");
    }
    bool done = false;
    for (long it = 0; it < kTcSpin && !done; it++) done = tc_bar_test(bar, 0);
    if (!done) {
        *err = 1;
        for (long it = 0; it < kTcSpin && !done; it++) done = tc_bar_test(bar, 0);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int ok = __syncthreads_and(done ? 1 : 0);
    if (ok) {
        const int i = row0 + warp * 32 + lane;
        TO *orow = out + (size_t)i * N;
        for (int c0 = 0; c0 < NP; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
                "%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                  "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                  "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (i >= n) continue;
            if constexpr (std::is_same<TO, bf16>::value) {
                // 8 outputs per 16-byte store (N is a multiple of 8)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int o0 = c0 + 8 * h;
                    if (o0 >= N) break;
                    __align__(16) bf16 v[8];
#pragma unroll
                    for (int e = 0; e < 8; e++)
                        v[e] = __float2bfloat16(tc_act(__uint_as_float(r[8 * h + e]) + b[o0 + e], act));
                    *reinterpret_cast<uint4 *>(orow + o0) = *reinterpret_cast<const uint4 *>(v);
                }
            } else {
                // 4 outputs per 16-byte store (N is a multiple of 4)
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const int o0 = c0 + 4 * h;
                    if (o0 >= N) break;
                    float4 v;
                    v.x = tc_act(__uint_as_float(r[4 * h + 0]) + b[o0 + 0], act);
                    v.y = tc_act(__uint_as_float(r[4 * h + 1]) + b[o0 + 1], act);
                    v.z = tc_act(__uint_as_float(r[4 * h + 2]) + b[o0 + 2], act);
                    v.w = tc_act(__uint_as_float(r[4 * h + 3]) + b[o0 + 3], act);
                    *reinterpret_cast<float4 *>(orow + o0) = v;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                     : "memory");
}

size_t tc_smem(int K, int NP) { return (size_t)(kTcRows + NP) * K * sizeof(bf16); }

// ---- the network's input graph on the device ---------------------------
// The normalised adjacency of the N^3 finite-volume operator from the cell
// conductivities kap (node i = (a0 N + a1) N + a2): the neighbours of i are
// i - N^2, i - N, i - 1, i + 1, i + N, i + N^2 (slots 0..5, ascending) where
// they lie in the grid; a face between a lower cell a and an upper cell b
// has t = 2 k_a k_b / (k_a + k_b); s_i = t_0 + ... + t_5 in slot order
// (absent slots 0); w_ij = t_ij / sqrt(s_i s_j) rounded to FP32.  These are
// the operations, in the same order, of the host construction, so the CSR
// is the same to the bit.
__global__ void grid_faces_kernel(int N, const double *__restrict__ kap, double *__restrict__ T,
                                  double *__restrict__ s, int32_t *__restrict__ deg) {
    const int64_t n = (int64_t)N * N * N;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a0 = (int)(i / ((int64_t)N * N)), a1 = (int)((i / N) % N), a2 = (int)(i % N);
    const int64_t step[6] = {-(int64_t)N * N, -(int64_t)N, -1, 1, N, (int64_t)N * N};
    const bool in[6] = {a0 > 0, a1 > 0, a2 > 0, a2 < N - 1, a1 < N - 1, a0 < N - 1};
    const double ki = kap[i];
    double acc = 0.0;
    int d = 0;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        double t = 0.0;
        if (in[j]) {
            const double kj = kap[i + step[j]];
            // slots 0-2: the neighbour is the lower cell; 3-5: this cell is
            t = j < 3 ? 2.0 * kj * ki / (kj + ki) : 2.0 * ki * kj / (ki + kj);
        }
        T[i * 6 + j] = t;
        acc += t;
        d += t > 0.0;
    }
    s[i] = acc;
    deg[i] = d;
}

__global__ void grid_fill_kernel(int N, const double *__restrict__ T, const double *__restrict__ s,
                                 const int32_t *__restrict__ rowptr, int32_t *__restrict__ col,
                                 float *__restrict__ w) {
    const int64_t n = (int64_t)N * N * N;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t step[6] = {-(int64_t)N * N, -(int64_t)N, -1, 1, N, (int64_t)N * N};
    int32_t q = rowptr[i];
    const double si = s[i];
#pragma unroll
    for (int j = 0; j < 6; j++) {
        const double t = T[i * 6 + j];
        if (t > 0.0) {
            const int64_t c = i + step[j];
            col[q] = (int32_t)c;
            w[q] = (float)(t / sqrt(si * s[c]));
            q++;
        }
    }
}

// ---- loss: G = Y^T Y (P x P), B = Y^T U (P x k), FP64 sums
__global__ void __launch_bounds__(kThreads)
gram_kernel(int n, int P, const float *__restrict__ Y, int k, const float *__restrict__ U,
            double *G, double *B) {
    extern __shared__ float sm[];
    const int R = 128;
    float *Ys = sm, *Us = sm + R * P;
    const int r0 = blockIdx.x * R;
    for (int t = threadIdx.x; t < R * P; t += blockDim.x) {
        const int i = r0 + t / P;
        Ys[t] = (i < n) ? Y[(size_t)i * P + t % P] : 0.f;
    }
    for (int t = threadIdx.x; t < R * k; t += blockDim.x) {
        const int i = r0 + t / k;
        Us[t] = (i < n) ? U[(size_t)i * k + t % k] : 0.f;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < P * (P + k); t += blockDim.x) {
        const int a = t / (P + k), c = t % (P + k);
        double acc = 0.0;
        if (c < P) {
            if (c < a) continue;                      // symmetric: upper part
            for (int r = 0; r < R; r++) acc += (double)Ys[r * P + a] * Ys[r * P + c];
            atomicAdd(G + a * P + c, acc);
        } else {
            const int bcol = c - P;
            for (int r = 0; r < R; r++) acc += (double)Ys[r * P + a] * Us[r * k + bcol];
            atomicAdd(B + a * k + bcol, acc);
        }
    }
}

// C = (G + eps tr(G)/P I)^{-1} B by Cholesky in one block (P <= 64);
// loss = 1 - trace(B^T C) / k.  G holds its upper triangle.
__global__ void small_solve_kernel(int P, int k, const double *G, const double *B, float *C,
                                   double *loss) {
    __shared__ double L[64 * 64];
    if (threadIdx.x == 0) {
        double tr = 0.0;
        for (int a = 0; a < P; a++) tr += G[a * P + a];
        const double eps = 1e-8 * tr / P + 1e-300;
        for (int a = 0; a < P; a++)
            for (int c = 0; c < P; c++) L[a * 64 + c] = (a <= c ? G[a * P + c] : G[c * P + a]) + (a == c ? eps : 0.0);
        for (int j = 0; j < P; j++) {
            double d = L[j * 64 + j];
            for (int t = 0; t < j; t++) d -= L[j * 64 + t] * L[j * 64 + t];
            d = sqrt(d > 0.0 ? d : 1e-300);
            L[j * 64 + j] = d;
            for (int i = j + 1; i < P; i++) {
                double s = L[i * 64 + j];
                for (int t = 0; t < j; t++) s -= L[i * 64 + t] * L[j * 64 + t];
                L[i * 64 + j] = s / d;
            }
        }
        double tr2 = 0.0;
        for (int b = 0; b < k; b++) {
            double z[64], x[64];
            for (int i = 0; i < P; i++) {
                double s = B[i * k + b];
                for (int t = 0; t < i; t++) s -= L[i * 64 + t] * z[t];
                z[i] = s / L[i * 64 + i];
            }
            for (int i = P - 1; i >= 0; i--) {
                double s = z[i];
                for (int t = i + 1; t < P; t++) s -= L[t * 64 + i] * x[t];
                x[i] = s / L[i * 64 + i];
            }
            for (int i = 0; i < P; i++) {
                tr2 += B[i * k + b] * x[i];
                C[i * k + b] = (float)x[i];
            }
        }
        *loss = 1.0 - tr2 / k;
    }
}

// dY[i, a] = -(2/k) sum_b (U[i, b] - sum_c Y[i, c] C[c, b]) C[a, b]
__global__ void dy_kernel(int n, int P, int k, const float *__restrict__ Y,
                          const float *__restrict__ U, const float *__restrict__ C, float *dY) {
    extern __shared__ float Cs[];
    for (int t = threadIdx.x; t < P * k; t += blockDim.x) Cs[t] = C[t];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float e[64];
    for (int b = 0; b < k; b++) {
        float s = U[(size_t)i * k + b];
        for (int c = 0; c < P; c++) s -= Y[(size_t)i * P + c] * Cs[c * k + b];
        e[b] = s;
    }
    const float sc = -2.f / k;
    for (int a = 0; a < P; a++) {
        float s = 0.f;
        for (int b = 0; b < k; b++) s += e[b] * Cs[a * k + b];
        dY[(size_t)i * P + a] = sc * s;
    }
}

// Adam on the FP32 weights, refreshing their BF16 copies
__global__ void adam_kernel(int64_t cnt, float *p, const float *g, float *m, float *v, float lr,
                            float b1, float b2, float c1, float c2, float eps, bf16 *pb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16(pi);
    }
}

__global__ void to_bf16_kernel(int64_t cnt, const float *src, bf16 *dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16(src[i]);
}

template <class T>
T *dalloc(size_t cnt) {
    void *p = nullptr;
    if (cudaMalloc(&p, (cnt ? cnt : 1) * sizeof(T)) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    return (T *)p;
}

}  // namespace

struct speigs_mpnn_s {
    int F = 0, H = 64, L = 4, P = 0;
    int64_t nparam = 0;
    std::vector<int64_t> woff, boff;   // per layer (0 = input, 1..L, L+1 = output)
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    bf16 *pb = nullptr;
    int64_t step = 0;
    int64_t ncap = 0;
    bf16 *Hs = nullptr, *Ms = nullptr;   // (L+1) x n x H, L x n x H
    float *Y = nullptr, *dY = nullptr, *dH = nullptr, *dH2 = nullptr, *dM = nullptr;
    double *G = nullptr, *B = nullptr, *loss = nullptr;
    float *C = nullptr;
    int kcap = 0;
    // dense layers of the forward pass on the tensor cores (tcgen05) where
    // their shapes allow it; 0 selects the FP32-FMA kernels throughout
    int tensor_cores = 1;
    // set by a tensor-core wait that ran out; mapped page-locked memory, so
    // the host reads it without synchronising the stream
    int *err_h = nullptr, *err_d = nullptr;
    // scratch of the device grid graph: face values (6 a node), node sums,
    // degrees and the scan's temporary storage
    double *gT = nullptr, *gs = nullptr;
    int32_t *gdeg = nullptr;
    void *gscan = nullptr;
    size_t gscan_bytes = 0;
    int64_t gcap = 0;
    ~speigs_mpnn_s() {
        void *ptrs[] = {p, g, m, v, pb, Hs, Ms, Y, dY, dH, dH2, dM, G, B, loss, C, gT, gs, gdeg,
                        gscan};
        for (void *q : ptrs)
            if (q) cudaFree(q);
        if (err_h) cudaFreeHost(err_h);
    }
    int layer_in(int l) const { return l == 0 ? F : (l <= L ? 2 * H : H); }
    int layer_out(int l) const { return l <= L ? H : P; }
    int reserve(int64_t n, int k) {
        if (n <= ncap && k <= kcap) return 0;
        void *ptrs[] = {Hs, Ms, Y, dY, dH, dH2, dM, G, B, loss, C};
        for (void *q : ptrs)
            if (q) cudaFree(q);
        ncap = std::max(n, ncap);
        kcap = std::max(k, kcap);
        Hs = dalloc<bf16>((size_t)(L + 1) * ncap * H);
        Ms = dalloc<bf16>((size_t)L * ncap * H);
        Y = dalloc<float>((size_t)ncap * P);
        dY = dalloc<float>((size_t)ncap * P);
        dH = dalloc<float>((size_t)ncap * H);
        dH2 = dalloc<float>((size_t)ncap * H);
        dM = dalloc<float>((size_t)ncap * H);
        G = dalloc<double>((size_t)P * P);
        B = dalloc<double>((size_t)P * std::max(kcap, 1));
        loss = dalloc<double>(1);
        C = dalloc<float>((size_t)P * std::max(kcap, 1));
        if (!Hs || !Ms || !Y || !dY || !dH || !dH2 || !dM || !G || !B || !loss || !C)
            return SPEIGS_ERR_MEM;
        return 0;
    }
};

namespace {

size_t dense_smem(int K, int N, bool bwd) {
    size_t f = (size_t)kRows * (K + 1) + (size_t)N * (K + 1) + (bwd ? (size_t)kRows * (N + 1) : 0);
    return f * sizeof(float);
}

void set_smem_limits() {
    const int big = 200 * 1024;
    cudaFuncSetAttribute(gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_fwd_kernel<float, bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_fwd_kernel<bf16, bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_fwd_kernel<bf16, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_bwd_kernel<float, bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_bwd_kernel<bf16, bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_bwd_kernel<bf16, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(dense_fwd_tc_kernel<bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)tc_smem(128, 64));
    cudaFuncSetAttribute(dense_fwd_tc_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)tc_smem(128, 64));
}

bool aligned16(const void *q) { return ((uintptr_t)q & 15u) == 0; }

// out = act(b + [X1, X2] W^T) for BF16 X1/X2 (node-major, K1 and K2 wide):
// the tensor-core kernel when the network allows it and the shapes and
// addresses fit its 16-byte pieces, else the FP32-FMA kernel
template <class TO>
void dense_fwd(const speigs_mpnn_s *net, int n, int K1, const bf16 *X1, int K2, const bf16 *X2,
               int N, const bf16 *W, const float *b, int act, TO *out, cudaStream_t st) {
    const int K = K1 + K2;
    const int vec = 16 / (int)sizeof(TO);
    const bool tc = net->tensor_cores && K1 % 8 == 0 && K2 % 8 == 0 && K % 16 == 0 && K <= 128 &&
                    N <= 64 && N % vec == 0 && aligned16(X1) && (K2 == 0 || aligned16(X2)) &&
                    aligned16(W) && aligned16(out);
    if (tc) {
        const int NP = (N + 15) & ~15;
        dense_fwd_tc_kernel<TO><<<(n + kTcRows - 1) / kTcRows, kTcThreads, tc_smem(K, NP), st>>>(
            n, K1, X1, K2, X2, N, NP, W, b, act, out, net->err_d);
    } else {
        dense_fwd_kernel<bf16, TO><<<(n + kRows - 1) / kRows, kThreads, dense_smem(K, N, false), st>>>(
            n, K1, X1, K2, X2, N, W, b, act, out);
    }
    spx::note_launch();
}

// forward pass keeping the activations; Y (FP32) in net->Y
void forward(speigs_mpnn_s *net, int n, const int32_t *rp, const int32_t *ci, const float *w,
             const float *X, cudaStream_t st) {
    const int H = net->H, L = net->L;
    const int nb = (n + kRows - 1) / kRows;
    const int sb = (n + 7) / 8;
    bf16 *Hl = net->Hs;
    dense_fwd_kernel<float, bf16><<<nb, kThreads, dense_smem(net->F, H, false), st>>>(
        n, net->F, X, 0, nullptr, H, net->pb + net->woff[0], net->p + net->boff[0], 1, Hl);
    spx::note_launch();
    for (int l = 1; l <= L; l++) {
        bf16 *Hp = net->Hs + (size_t)(l - 1) * n * H, *Hn = net->Hs + (size_t)l * n * H;
        bf16 *Ml = net->Ms + (size_t)(l - 1) * n * H;
        spmm_kernel<bf16, bf16><<<sb, 256, 0, st>>>(n, H, rp, ci, w, Hp, Ml, 0);
        spx::note_launch();
        dense_fwd<bf16>(net, n, H, Hp, H, Ml, H, net->pb + net->woff[l], net->p + net->boff[l], 1,
                        Hn, st);
    }
    dense_fwd<float>(net, n, H, net->Hs + (size_t)L * n * H, 0, nullptr, net->P,
                     net->pb + net->woff[L + 1], net->p + net->boff[L + 1], 0, net->Y, st);
}

}  // namespace

extern "C" {

int speigs_b200_mpnn_create(int nfeat, int hidden, int layers, int nout, uint64_t seed,
                            speigs_mpnn *out) {
    if (!out || nfeat < 1 || nfeat > 64 || hidden != 64 || layers < 0 || layers > 8 || nout < 1 ||
        nout > 64)
        return SPEIGS_ERR_ARG;
    *out = nullptr;
    speigs_mpnn_s *net = new (std::nothrow) speigs_mpnn_s;
    if (!net) return SPEIGS_ERR_MEM;
    net->F = nfeat;
    net->H = hidden;
    net->L = layers;
    net->P = nout;
    int64_t off = 0;
    for (int l = 0; l <= layers + 1; l++) {
        net->woff.push_back(off);
        off += (int64_t)net->layer_out(l) * net->layer_in(l);
        net->boff.push_back(off);
        off += net->layer_out(l);
    }
    net->nparam = off;
    // Xavier-uniform weights from a seeded xorshift64* stream, zero biases
    std::vector<float> hp(off, 0.f);
    uint64_t s = seed ? seed : 88172645463325252ULL;
    auto uni = [&]() {
        s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
        return (double)((s * 0x2545F4914F6CDD1DULL) >> 11) / 9007199254740992.0;
    };
    for (int l = 0; l <= layers + 1; l++) {
        const int fi = net->layer_in(l), fo = net->layer_out(l);
        const double a = std::sqrt(6.0 / (fi + fo)) * (l == layers + 1 ? 0.1 : 1.0);
        for (int64_t t = 0; t < (int64_t)fi * fo; t++) hp[net->woff[l] + t] = (float)((2.0 * uni() - 1.0) * a);
    }
    net->p = dalloc<float>(off);
    net->g = dalloc<float>(off);
    net->m = dalloc<float>(off);
    net->v = dalloc<float>(off);
    net->pb = dalloc<bf16>(off);
    if (!net->p || !net->g || !net->m || !net->v || !net->pb) { delete net; return SPEIGS_ERR_MEM; }
    cudaMemcpy(net->p, hp.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
    cudaMemset(net->m, 0, sizeof(float) * off);
    cudaMemset(net->v, 0, sizeof(float) * off);
    cudaMemset(net->g, 0, sizeof(float) * off);
    to_bf16_kernel<<<64, 256>>>(off, net->p, net->pb);
    spx::note_launch();
    if (cudaHostAlloc((void **)&net->err_h, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&net->err_d, net->err_h, 0) != cudaSuccess) {
        cudaGetLastError();
        delete net;
        return SPEIGS_ERR_MEM;
    }
    *net->err_h = 0;
    set_smem_limits();
    if (cudaDeviceSynchronize() != cudaSuccess) { cudaGetLastError(); delete net; return SPEIGS_ERR_INTERNAL; }
    *out = net;
    return SPEIGS_OK;
}

void speigs_b200_mpnn_destroy(speigs_mpnn net) { delete net; }

int speigs_b200_mpnn_grid_graph(speigs_mpnn net, int N, const double *kap, int32_t *rowptr,
                                int32_t *col, float *w, void *stream) {
    if (!net || N < 1 || (int64_t)N * N * N > INT32_MAX / 6 || !kap || !rowptr || !col || !w)
        return SPEIGS_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = (int64_t)N * N * N;
    if (n > net->gcap) {
        void *old[] = {net->gT, net->gs, net->gdeg, net->gscan};
        for (void *q : old)
            if (q) cudaFree(q);
        net->gT = dalloc<double>((size_t)n * 6);
        net->gs = dalloc<double>((size_t)n);
        net->gdeg = dalloc<int32_t>((size_t)n);
        net->gscan_bytes = 0;
        cub::DeviceScan::InclusiveSum(nullptr, net->gscan_bytes, net->gdeg, rowptr + 1, (int)n, st);
        net->gscan = net->gscan_bytes ? (void *)dalloc<unsigned char>(net->gscan_bytes) : nullptr;
        net->gcap = (net->gT && net->gs && net->gdeg && (net->gscan || !net->gscan_bytes)) ? n : 0;
        if (!net->gcap) return SPEIGS_ERR_MEM;
    }
    const int tb = 256, nb = (int)((n + tb - 1) / tb);
    grid_faces_kernel<<<nb, tb, 0, st>>>(N, kap, net->gT, net->gs, net->gdeg);
    cudaMemsetAsync(rowptr, 0, sizeof(int32_t), st);
    size_t tmp = net->gscan_bytes;
    cub::DeviceScan::InclusiveSum(net->gscan, tmp, net->gdeg, rowptr + 1, (int)n, st);
    grid_fill_kernel<<<nb, tb, 0, st>>>(N, net->gT, net->gs, rowptr, col, w);
    spx::note_launch(3);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { spx::set_last_error_text(cudaGetErrorString(e)); return SPEIGS_ERR_INTERNAL; }
    return SPEIGS_OK;
}

int speigs_b200_mpnn_tensor_cores(speigs_mpnn net, int on) {
    if (!net) return SPEIGS_ERR_ARG;
    const int was = net->tensor_cores;
    if (on >= 0) net->tensor_cores = on ? 1 : 0;
    return was;
}

int speigs_b200_mpnn_params(speigs_mpnn net, float *host, int64_t *count, int set) {
    if (!net || !count) return SPEIGS_ERR_ARG;
    if (!host) { *count = net->nparam; return SPEIGS_OK; }
    if (*count < net->nparam) return SPEIGS_ERR_ARG;
    if (set) {
        cudaMemcpy(net->p, host, sizeof(float) * net->nparam, cudaMemcpyHostToDevice);
        to_bf16_kernel<<<64, 256>>>(net->nparam, net->p, net->pb);
        spx::note_launch();
    } else {
        cudaMemcpy(host, net->p, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost);
    }
    *count = net->nparam;
    return cudaDeviceSynchronize() == cudaSuccess ? SPEIGS_OK : SPEIGS_ERR_INTERNAL;
}

int speigs_b200_mpnn_grads(speigs_mpnn net, float *host) {
    if (!net || !host) return SPEIGS_ERR_ARG;
    cudaMemcpy(host, net->g, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost);
    return cudaDeviceSynchronize() == cudaSuccess ? SPEIGS_OK : SPEIGS_ERR_INTERNAL;
}

int speigs_b200_mpnn_forward(speigs_mpnn net, int64_t n, const int32_t *rowptr, const int32_t *col,
                             const float *w, const float *X, float *Y, void *stream) {
    if (!net || n <= 0 || n > INT32_MAX || !rowptr || !col || !w || !X || !Y) return SPEIGS_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (*(volatile int *)net->err_h) {
        spx::set_last_error_text("mpnn: a tensor-core wait of an earlier call ran out");
        return SPEIGS_ERR_INTERNAL;
    }
    if (net->reserve(n, 1)) return SPEIGS_ERR_MEM;
    forward(net, (int)n, rowptr, col, w, X, st);
    cudaMemcpyAsync(Y, net->Y, sizeof(float) * (size_t)n * net->P, cudaMemcpyDeviceToDevice, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { spx::set_last_error_text(cudaGetErrorString(e)); return SPEIGS_ERR_INTERNAL; }
    return SPEIGS_OK;
}

int speigs_b200_mpnn_train_step(speigs_mpnn net, int64_t n, const int32_t *rowptr,
                                const int32_t *col, const float *w, const float *X,
                                const float *U, int k, float lr, double *loss, void *stream) {
    if (!net || n <= 0 || n > INT32_MAX || !rowptr || !col || !w || !X || !U || k < 1 || k > 64)
        return SPEIGS_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (net->reserve(n, k)) return SPEIGS_ERR_MEM;
    const int H = net->H, L = net->L, P = net->P, nn = (int)n;
    const int nb = (nn + kRows - 1) / kRows, sb = (nn + 7) / 8;
    forward(net, nn, rowptr, col, w, X, st);
    // loss and dL/dY
    cudaMemsetAsync(net->G, 0, sizeof(double) * P * P, st);
    cudaMemsetAsync(net->B, 0, sizeof(double) * P * k, st);
    gram_kernel<<<(nn + 127) / 128, kThreads, sizeof(float) * 128 * (P + k), st>>>(nn, P, net->Y, k, U,
                                                                               net->G, net->B);
    small_solve_kernel<<<1, 32, 0, st>>>(P, k, net->G, net->B, net->C, net->loss);
    dy_kernel<<<(nn + 127) / 128, 128, sizeof(float) * P * k, st>>>(nn, P, k, net->Y, U, net->C, net->dY);
    spx::note_launch(3);
    // backward
    cudaMemsetAsync(net->g, 0, sizeof(float) * net->nparam, st);
    bf16 *HL = net->Hs + (size_t)L * nn * H;
    dense_bwd_kernel<bf16, float><<<nb, kThreads, dense_smem(H, P, true), st>>>(
        nn, H, HL, 0, nullptr, P, net->pb + net->woff[L + 1], 0, net->Y, net->dY, net->dH, nullptr,
        0, net->g + net->woff[L + 1], net->g + net->boff[L + 1]);
    spx::note_launch();
    for (int l = L; l >= 1; l--) {
        bf16 *Hp = net->Hs + (size_t)(l - 1) * nn * H, *Hn = net->Hs + (size_t)l * nn * H;
        bf16 *Ml = net->Ms + (size_t)(l - 1) * nn * H;
        // dH currently holds dL/dh_l; produce dL/dh_{l-1} (direct part) and dL/dm_l
        float *dHn = net->dH;
        dense_bwd_kernel<bf16, bf16><<<nb, kThreads, dense_smem(2 * H, H, true), st>>>(
            nn, H, Hp, H, Ml, H, net->pb + net->woff[l], 1, Hn, dHn, net->dH2, net->dM, 0,
            net->g + net->woff[l], net->g + net->boff[l]);
        // dL/dh_{l-1} = direct part + A^T dL/dm_l (A symmetric)
        spmm_kernel<float, float><<<sb, 256, 0, st>>>(nn, H, rowptr, col, w, net->dM, net->dH2, 1);
        std::swap(net->dH, net->dH2);
        spx::note_launch(2);
    }
    dense_bwd_kernel<float, bf16><<<nb, kThreads, dense_smem(net->F, H, true), st>>>(
        nn, net->F, X, 0, nullptr, H, net->pb + net->woff[0], 1, net->Hs, net->dH, nullptr,
        nullptr, 0, net->g + net->woff[0], net->g + net->boff[0]);
    spx::note_launch();
    if (lr > 0.f) {
        net->step++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
        adam_kernel<<<256, 256, 0, st>>>(net->nparam, net->p, net->g, net->m, net->v, lr, b1, b2, c1,
                                         c2, 1e-8f, net->pb);
        spx::note_launch();
    }
    double hl = 0.0;
    cudaMemcpyAsync(&hl, net->loss, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { spx::set_last_error_text(cudaGetErrorString(e)); return SPEIGS_ERR_INTERNAL; }
    if (*(volatile int *)net->err_h) {
        spx::set_last_error_text("mpnn: a tensor-core wait ran out");
        return SPEIGS_ERR_INTERNAL;
    }
    if (loss) *loss = hl;
    return SPEIGS_OK;
}

}  // extern "C"
