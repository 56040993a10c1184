// vx_clusters.cu — rebuild_clusters (src/solver.rs:828-858) on the device.
//
// Connected components of the bond graph by lock-free union-find: every bond
// links the larger of its endpoints' roots under the smaller with atomicCAS
// (parents only ever decrease, so path halving by plain stores is safe), then
// a read-only walk gives every REV its root, the smallest REV of its component. The
// reference numbers clusters in the order its HashMap first sees them while
// walking REVs by index, skipping kinematic REVs: a component's id is the
// number of components whose first non-kinematic REV comes earlier. That is an
// exclusive prefix sum over "REV i is its component's first non-kinematic REV"
// flags, so the ids are the reference's bits, independent of thread timing.
#include "vx_device.cuh"
#include "vx_kernels.h"

namespace vx {

namespace {

constexpr unsigned kScanBlock = 1024;  // REVs per scan block (256 threads x 4)
constexpr unsigned kHookRetries = 1u << 16;

__device__ __forceinline__ uint32_t find_root(uint32_t* parent, uint32_t x) {
    uint32_t p = __ldcg(parent + x);
    while (p != x) {  // indices strictly decrease along the path: the loop ends
        const uint32_t g = __ldcg(parent + p);
        if (g != p) __stcg(parent + x, g);  // path halving; g < p, so parents keep decreasing
        x = p;
        p = g;
    }
    return x;
}

__global__ void k_cluster_init(uint32_t n, uint32_t* __restrict__ parent, uint32_t* __restrict__ first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    parent[i] = i;
    first[i] = VX_EMPTY_U32;
}

__global__ void k_cluster_hook(uint32_t n, const uint32_t* __restrict__ nbr, uint32_t* parent,
                               uint32_t* __restrict__ err) {
    const size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= 3 * (size_t)n) return;
    const uint32_t j = nbr[e];
    if (j == VX_EMPTY_U32 || j >= n) return;
    const uint32_t i = (uint32_t)(e % n);
    for (unsigned tries = 0; tries < kHookRetries; ++tries) {
        const uint32_t ri = find_root(parent, i), rj = find_root(parent, j);
        if (ri == rj) return;
        const uint32_t lo = ri < rj ? ri : rj, hi = ri < rj ? rj : ri;
        if (atomicCAS(parent + hi, hi, lo) == hi) return;  // else hi was linked meanwhile: retry
    }
    atomicExch(err, 1u);
}

// After the hooks: each REV's root by a read-only walk (no store races with
// other walks), and each component's first non-kinematic REV.
__global__ void k_cluster_roots(uint32_t n, const uint32_t* __restrict__ parent, const uint8_t* __restrict__ kin,
                                uint32_t* __restrict__ root, uint32_t* __restrict__ first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x = i, p = parent[i];
    while (p != x) {
        x = p;
        p = parent[p];
    }
    root[i] = x;
    if (!kin[i]) atomicMin(first + x, i);
}

// flags[i] = 1 where i is the first non-kinematic REV of its component; per
// scan block, the inclusive block total goes to bsum[block].
__global__ void __launch_bounds__(256) k_cluster_flags(uint32_t n, const uint32_t* root, const uint32_t* first,
                                                       const uint8_t* __restrict__ kin, uint32_t* __restrict__ scan,
                                                       uint32_t* __restrict__ bsum) {
    __shared__ uint32_t warp_tot[8];
    const uint32_t base = blockIdx.x * kScanBlock + threadIdx.x * 4;
    uint32_t f[4], local = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = base + k;
        f[k] = 0;
        if (i < n && !kin[i]) f[k] = first[root[i]] == i ? 1u : 0u;
        local += f[k];
    }
    // exclusive scan of the per-thread totals inside the block
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += v;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (unsigned w = 0; w < warp; ++w) before += warp_tot[w];
    uint32_t run = before + incl - local;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = base + k;
        if (i < n) scan[i] = run;
        run += f[k];
    }
    if (threadIdx.x == blockDim.x - 1) bsum[blockIdx.x] = before + incl;
}

// Exclusive scan of the block totals by one block; bsum[nb] = grand total.
__global__ void __launch_bounds__(1024) k_cluster_block_scan(uint32_t nb, uint32_t* bsum) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t lo = 0; lo < nb; lo += blockDim.x) {
        const uint32_t k = lo + threadIdx.x;
        const uint32_t v = k < nb ? bsum[k] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t before = 0;
        for (unsigned w = 0; w < warp; ++w) before += warp_tot[w];
        const uint32_t c0 = carry;
        if (k < nb) bsum[k] = c0 + before + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c0 + before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void k_cluster_ids(uint32_t n, const uint32_t* root, const uint32_t* first,
                              const uint8_t* __restrict__ kin, const uint32_t* __restrict__ scan,
                              const uint32_t* __restrict__ bsum, uint32_t* __restrict__ clusters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kin[i]) {
        clusters[i] = VX_EMPTY_U32;
        return;
    }
    const uint32_t f = first[root[i]];
    clusters[i] = scan[f] + bsum[f / kScanBlock];
}

}  // namespace

cudaError_t launch_rebuild_clusters(vx_scene* s) {
    const uint32_t n = s->n;
    cudaError_t e = cudaMemsetAsync(s->cl_err, 0, sizeof(uint32_t), s->stream);
    if (e != cudaSuccess || n == 0) return e;
    const unsigned g = (n + 255) / 256, nb = (n + kScanBlock - 1) / kScanBlock;
    k_cluster_init<<<g, 256, 0, s->stream>>>(n, s->cl_parent, s->cl_first);
    k_cluster_hook<<<(unsigned)((3 * (size_t)n + 255) / 256), 256, 0, s->stream>>>(n, s->nbr, s->cl_parent, s->cl_err);
    k_cluster_roots<<<g, 256, 0, s->stream>>>(n, s->cl_parent, s->kin, s->cl_root, s->cl_first);
    k_cluster_flags<<<nb, 256, 0, s->stream>>>(n, s->cl_root, s->cl_first, s->kin, s->cl_scan, s->cl_bsum);
    k_cluster_block_scan<<<1, 1024, 0, s->stream>>>(nb, s->cl_bsum);
    k_cluster_ids<<<g, 256, 0, s->stream>>>(n, s->cl_root, s->cl_first, s->kin, s->cl_scan, s->cl_bsum,
                                            s->clusters);
    return cudaGetLastError();
}

uint32_t cluster_scan_blocks(uint32_t n) { return (n + kScanBlock - 1) / kScanBlock; }

}  // namespace vx

using namespace vx;

extern "C" int32_t vx_scene_rebuild_clusters(vx_scene* s, uint32_t* clusters, uint32_t* out_count) {
    clear_error();
    if (!s) {
        set_error("vx_scene_rebuild_clusters: null scene");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    cudaError_t e = launch_rebuild_clusters(s);
    uint32_t tail[2] = {0, 0};
    const uint32_t nb = cluster_scan_blocks(s->n);
    if (e == cudaSuccess && s->n)
        e = cudaMemcpyAsync(&tail[0], s->cl_bsum + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[1], s->cl_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && clusters && s->n)
        e = cudaMemcpyAsync(clusters, s->clusters, s->n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        set_error("vx_scene_rebuild_clusters: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    if (tail[1]) {
        set_error("vx_scene_rebuild_clusters: a union did not settle within its retry bound");
        return VX_TIMEOUT;
    }
    if (out_count) *out_count = tail[0];
    return VX_OK;
}
