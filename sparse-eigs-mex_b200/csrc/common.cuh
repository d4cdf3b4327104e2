// Shared device helpers for the speigs B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SPX_DEV __device__ __forceinline__

namespace spx {

constexpr int kWarp = 32;

SPX_DEV double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; every thread gets the result.  `sh` holds >= 32 doubles.
SPX_DEV double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < (unsigned)nw) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// Block-wide sums of eight values at once.  Inside a warp, three exchange
// steps (4 + 2 + 1 shuffles) leave lane L holding column L & 7 summed over
// the eight lanes that share bits 3-4 of L; two more shuffles finish the
// warp.  The warps' totals meet in `sh` (>= 8 doubles per warp); thread
// q < 8 returns the block total of column q (the other threads return 0).
SPX_DEV double block_sum8(double (&v)[8], double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    double p4[4], p2[2];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const bool hi = lane & 4;
        const double send = hi ? v[m] : v[m + 4];
        const double keep = hi ? v[m + 4] : v[m];
        p4[m] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
#pragma unroll
    for (int m = 0; m < 2; m++) {
        const bool hi = lane & 2;
        const double send = hi ? p4[m] : p4[m + 2];
        const double keep = hi ? p4[m + 2] : p4[m];
        p2[m] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    double t;
    {
        const bool hi = lane & 1;
        const double send = hi ? p2[0] : p2[1];
        const double keep = hi ? p2[1] : p2[0];
        t = keep + __shfl_xor_sync(0xffffffffu, send, 1);
    }
    t += __shfl_xor_sync(0xffffffffu, t, 8);
    t += __shfl_xor_sync(0xffffffffu, t, 16);
    __syncthreads();
    if (lane < 8) sh[wid * 8 + lane] = t;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 8)
        for (int w = 0; w < nw; w++) r += sh[w * 8 + threadIdx.x];
    return r;
}

// Index of the last element of a sorted prefix array <= key (binary search).
SPX_DEV int upper_index(const int64_t *prefix, int n, int64_t key) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= key) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace spx
