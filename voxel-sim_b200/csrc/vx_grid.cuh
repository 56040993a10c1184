// vx_grid.cuh — grid-wide synchronisation of the cooperative (persistent)
// inner-solve kernels: acquire/release accesses and a deterministic grid
// reduction that doubles as a grid barrier.
#pragma once

#include "vx_device.cuh"

namespace vx {

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block-wide sum of NV values, published as this block's partials, then the
// grid-wide totals once all G blocks have arrived at reduction number `seq`
// (the arrival counter only grows: reduction seq is complete at seq * G).
// The __syncthreads before the release makes every thread's earlier global
// stores part of what the release publishes; the acquire by lane 0, then
// __syncwarp and the final __syncthreads, order every thread's later loads
// after the other blocks' released stores. One warp sums the G partials in
// block order, so every block gets the same bits. Returns false (in every
// thread) when a wait ran out here or in another block.
// A provides: part (double [NV slots][G]), count (u64 arrivals), err (int32),
// spin_limit (polls before giving up).
template <int NV, class A>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], const int (&slot)[NV], const A& a,
                                           unsigned long long seq, double (*sh)[32], double* tot, int* s_ok,
                                           double (&out)[NV]) {
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5, G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        double b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) b[k] = warp_sum(lane < nw ? sh[k][lane] : 0.0);
        int ok = 1;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.part[(size_t)slot[k] * G + blockIdx.x] = b[k];
            red_release_add_u64(a.count, 1ull);
            const unsigned long long target = seq * G;
            unsigned long long spins = 0;
            while (ld_acquire_u64(a.count) < target) {
                if (++spins >= a.spin_limit || ((spins & 63) == 0 && *(volatile int32_t*)a.err)) {
                    ok = 0;
                    break;
                }
            }
            if (!ok) atomicExch(a.err, 1);
            else if (*(volatile int32_t*)a.err) ok = 0;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        double t[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = 0.0;
        if (ok) {
            for (unsigned blk = lane; blk < G; blk += 32) {
#pragma unroll
                for (int k = 0; k < NV; ++k) t[k] += __ldcg(a.part + (size_t)slot[k] * G + blk);
            }
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = warp_sum(t[k]);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) tot[k] = t[k];
            *s_ok = ok;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = tot[k];
    return *s_ok != 0;
}

// grid_reduce in two halves, so that a block can work between its arrival
// and the wait: grid_arrive sums the block's NV values and publishes them
// (the __syncthreads in it also makes this block's shared-memory stores
// visible to all its threads); grid_complete waits for every block's arrival
// at reduction `seq` and returns the totals, in the same bits as grid_reduce.
// Between the two a block may not write a partial row or `sh`.
template <int NV, class A>
__device__ __forceinline__ void grid_arrive(double (&v)[NV], const int (&slot)[NV], const A& a, double (*sh)[32]) {
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5, G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        double b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) b[k] = warp_sum(lane < nw ? sh[k][lane] : 0.0);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.part[(size_t)slot[k] * G + blockIdx.x] = b[k];
            red_release_add_u64(a.count, 1ull);
        }
    }
}

template <int NV, class A>
__device__ __forceinline__ bool grid_complete(const int (&slot)[NV], const A& a, unsigned long long seq, double* tot,
                                             int* s_ok, double (&out)[NV]) {
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, G = gridDim.x;
    if (warp == 0) {
        int ok = 1;
        if (lane == 0) {
            const unsigned long long target = seq * G;
            unsigned long long spins = 0;
            while (ld_acquire_u64(a.count) < target) {
                if (++spins >= a.spin_limit || ((spins & 63) == 0 && *(volatile int32_t*)a.err)) {
                    ok = 0;
                    break;
                }
            }
            if (!ok) atomicExch(a.err, 1);
            else if (*(volatile int32_t*)a.err) ok = 0;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        double t[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = 0.0;
        if (ok) {
            for (unsigned blk = lane; blk < G; blk += 32) {
#pragma unroll
                for (int k = 0; k < NV; ++k) t[k] += __ldcg(a.part + (size_t)slot[k] * G + blk);
            }
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = warp_sum(t[k]);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) tot[k] = t[k];
            *s_ok = ok;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = tot[k];
    return *s_ok != 0;
}

// grid_reduce for blocks that work for different problems (the slots of a
// pool): the NV values are summed over the blocks [fb, fb + nb) of this block's
// own problem, in block order, and `act` over all G blocks (a count of blocks
// still at work, which tells every block when to stop). With fb = 0 and nb = G
// the NV sums are grid_reduce's bits. Partial rows: slot[k] for the NV values,
// act_row for act (act_row < 0: no act value). A row may only be written again
// by a reduction that has a grid barrier between it and this one's reads: a
// block past this barrier could otherwise overwrite a row another block has
// not read yet. A as for grid_reduce.
template <int NV, class A>
__device__ __forceinline__ bool grid_reduce_ranged(double (&v)[NV], double act, const int (&slot)[NV], int act_row,
                                                   const A& a, unsigned long long seq, uint32_t fb, uint32_t nb,
                                                   double (*sh)[32], double* tot, int* s_ok, double (&out)[NV],
                                                   double* act_total) {
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5, G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        double b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) b[k] = warp_sum(lane < nw ? sh[k][lane] : 0.0);
        int ok = 1;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.part[(size_t)slot[k] * G + blockIdx.x] = b[k];
            if (act_row >= 0) a.part[(size_t)act_row * G + blockIdx.x] = act;
            red_release_add_u64(a.count, 1ull);
            const unsigned long long target = seq * G;
            unsigned long long spins = 0;
            while (ld_acquire_u64(a.count) < target) {
                if (++spins >= a.spin_limit || ((spins & 63) == 0 && *(volatile int32_t*)a.err)) {
                    ok = 0;
                    break;
                }
            }
            if (!ok) atomicExch(a.err, 1);
            else if (*(volatile int32_t*)a.err) ok = 0;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        double t[NV], ta = 0.0;
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = 0.0;
        if (ok) {
            for (unsigned blk = lane; blk < nb; blk += 32) {
#pragma unroll
                for (int k = 0; k < NV; ++k) t[k] += __ldcg(a.part + (size_t)slot[k] * G + fb + blk);
            }
            if (act_row >= 0)
                for (unsigned blk = lane; blk < G; blk += 32) ta += __ldcg(a.part + (size_t)act_row * G + blk);
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = warp_sum(t[k]);
        ta = warp_sum(ta);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) tot[k] = t[k];
            tot[NV] = ta;
            *s_ok = ok;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = tot[k];
    *act_total = tot[NV];
    return *s_ok != 0;
}

}  // namespace vx
