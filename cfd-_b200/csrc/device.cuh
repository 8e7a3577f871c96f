// device.cuh - device-side helpers shared by the kernels: reductions, the
// last-block-done pattern, ordered bit-pattern max for non-negative doubles.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfd2d_b200.h"
#include "cellmath.cuh"

namespace cfd {

constexpr int kBlock = 256;

// max of non-negative doubles through their bit patterns; a NaN (positive after
// fabs) has a larger pattern than +inf, so NaN propagates like numpy's max.
__device__ __forceinline__ unsigned long long dbits(double x) {
    return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
    return __longlong_as_double((long long)b);
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double x) {
    atomicMax(slot, dbits(x));
}
// min over non-negative doubles (used for min nu_eff)
__device__ __forceinline__ void atomic_min_nonneg(unsigned long long* slot, double x) {
    atomicMin(slot, dbits(x));
}

// warp tree sum, fixed order (deterministic)
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = npmax(x, __shfl_down_sync(0xffffffffu, x, o));
    return x;
}

// Block sum of K values per thread; result valid in thread 0. smem: K*32 doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* smem) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) smem[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = (lane < nw) ? smem[k * 32 + lane] : 0.0;
            v[k] = warp_sum(x);
        }
    }
    __syncthreads();
}

template <int K>
__device__ __forceinline__ void block_max(double (&v)[K], double* smem, double ident = 0.0) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_max(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) smem[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = (lane < nw) ? smem[k * 32 + lane] : ident;
            v[k] = warp_max(x);
        }
    }
    __syncthreads();
}

// Last-block-done: every block calls this after publishing its partials; returns
// true in exactly one block (the last to arrive), which then sees all partials.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

}  // namespace cfd
