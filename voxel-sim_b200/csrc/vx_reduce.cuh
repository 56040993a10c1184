// vx_reduce.cuh — single-pass deterministic grid reductions in FP64.
//
// Each block reduces its values (warp shuffles, then one warp over the warp
// sums) and writes one partial per value; the block that takes the last
// ticket of an atomic counter sums all partials in a fixed order and resets
// the counter. The result does not depend on block scheduling.
#pragma once

#include "vx_device.cuh"

namespace vx {

constexpr int kThreads = 256;

// ---- block / grid reduction ---------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*smem)[kThreads / 32]) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < (kThreads / 32) ? smem[k][lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Block partials -> partials[k * grid + block]; returns true in the last block
// to finish, where v[] (thread 0) then holds the grid totals.
template <int NV>
__device__ bool grid_sum(double (&v)[NV], double* partials, unsigned* counter) {
    __shared__ double smem[NV][kThreads / 32];
    __shared__ bool last;
    block_sum<NV>(v, smem);
    const unsigned grid = gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[(size_t)k * grid + blockIdx.x] = v[k];
        __threadfence();
        unsigned ticket = atomicAdd(counter, 1u);
        last = (ticket == grid - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double t[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        t[k] = 0.0;
        for (unsigned b = threadIdx.x; b < grid; b += kThreads) t[k] += __ldcg(&partials[(size_t)k * grid + b]);
    }
    block_sum<NV>(t, smem);
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = t[k];
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

}  // namespace vx
