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
