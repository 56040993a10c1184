// vx_pool.cu — many scenes resident in one device arena, solved together.
//
// A pool reserves a capacity of REVs in 256-REV tiles. Each resident scene
// (a slot) occupies a contiguous, tile-aligned range; the REVs that pad its
// last tile are inert (kinematic, no bonds). All scenes share one index space,
// so the per-REV and per-bond kernels of a single scene (rotation fit,
// assembly, stress) run unchanged over the whole arena, skipping tiles of
// slots that are not part of the call.
//
// The solve is the FP32-inner / FP64-refinement form of vx_pcg.cu with every
// scalar kept per slot. A tile never spans two slots, so each tile's partial
// sums belong to one slot; small per-slot kernels (one warp per slot) add a
// slot's tile partials in tile order and derive its alpha, beta, convergence
// and iteration cap. A slot's arithmetic therefore does not depend on which
// other slots share the call: its result is bit-identical alone or in any
// mix. Converged slots drop out tile by tile while the others iterate.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_layout.cuh"
#include "vx_pcg_core.cuh"
#include "vx_reduce.cuh"

namespace vx {

struct PoolArgs {
    uint32_t tiles;
    uint32_t slots;
    const uint8_t* tile_on;
    const uint32_t* tile_scene;
    const uint32_t* slot_first;  // [slots] first tile
    const uint32_t* slot_tiles;  // [slots] tile count
    SlotState* st;
    double* tp;                  // [3][tiles] tile partials
    int32_t* active;             // slots still iterating in the inner solve
    int32_t* pending;            // slots that need an inner solve this outer step
    double tolerance;            // outer target
    double inner_tolerance;      // floor of the inner targets
    uint32_t max_iterations;     // inner iteration budget per slot and pass
    uint32_t max_outer;
};

}  // namespace vx

struct vx_pool {
    vx_scene s;  // the arena (n = capacity)
    uint32_t slots = 0;
    uint32_t tiles = 0;
    std::vector<uint32_t> owner;            // tile -> slot or VX_EMPTY
    std::vector<uint32_t> first, count, rev_n;
    std::vector<uint8_t> used;
    std::vector<uint8_t> h_tile_on;
    char* extra = nullptr;                  // pool-only device memory
    vx::SlotState* st = nullptr;            // device [slots]
    uint32_t* slot_first = nullptr;
    uint32_t* slot_tiles = nullptr;
    uint32_t* slot_revs = nullptr;          // device [slots]: REVs of the slot's scene
    int32_t* active = nullptr;
    int32_t* pending = nullptr;
    unsigned long long* angle = nullptr;    // [slots]
    vx::SlotState* h_st = nullptr;          // pinned [slots]
    int32_t* h_flag = nullptr;              // pinned [4]
    cudaGraphExec_t chunk = nullptr;
    // the slots packed into waves of the persistent inner solve: block rows
    // (first REV, REV count, slot, first block of the slot << 16 | its blocks)
    // and per wave its first row, block count and largest block
    bool waves_dirty = true;
    bool waves_ok = false;
    std::vector<uint4> wave_rows;
    std::vector<uint4> waves;               // (first row, blocks, largest block, 0)
    uint4* d_wave_rows = nullptr;
};

namespace vx {

int32_t scene_alloc(vx_scene* s, vx_ctx* ctx, uint32_t n, uint32_t material_count, size_t stage_revs);

// Pinned staging of a pool, in REVs: per-slot copies go through it in chunks.
constexpr size_t kPoolStageRevs = size_t(4) << 20;
void scene_release(vx_scene* s);

namespace {

constexpr int kPoolChunk = 16;

// Sum over one slot's tile partials by one warp, in tile order per lane and
// a fixed shuffle tree: the same for the slot whatever else is in the pool.
__device__ __forceinline__ double warp_total(const double* tp, uint32_t first, uint32_t cnt) {
    double v = 0.0;
    for (uint32_t k = threadIdx.x & 31; k < cnt; k += 32) v += __ldcg(tp + first + k);
    return warp_sum(v);
}

template <int NV>
__device__ __forceinline__ void tile_partial(double (&v)[NV], double* tp, uint32_t tiles, uint32_t t) {
    __shared__ double sh[NV][kThreads / 32];
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tp[(size_t)k * tiles + t] = v[k];
    }
}

__device__ __forceinline__ bool slot_iterating(const SlotState& S) { return S.enabled && S.inner_on && !S.done; }

// ---- tile kernels -------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_pool_zero(PoolArgs P, double* x64, uint32_t n) {
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        size_t i = (size_t)t * kThreads + threadIdx.x;
        x64[i] = 0.0, x64[n + i] = 0.0, x64[2 * (size_t)n + i] = 0.0;
    }
}

__global__ void __launch_bounds__(kThreads) k_pool_residual64(IterArgs<double> a, PoolArgs P,
                                                              const double* __restrict__ b, double* __restrict__ r_out) {
    const size_t n = a.n;
    const double* x = a.x;
    auto get = [&](uint32_t j) { return V3<double>{x[j], x[n + j], x[2 * n + j]}; };
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        const SlotState& S = P.st[P.tile_scene[t]];
        if (!S.enabled || S.outer_done) continue;
        const uint32_t i = t * kThreads + threadIdx.x;
        V3<double> y = apply_row<double>(a, i, get(i), get);
        V3<double> bb = load_v(b, n, i);
        V3<double> r = {bb.x - y.x, bb.y - y.y, bb.z - y.z};
        store_v(r_out, n, i, r);
        double v[2] = {r.x * r.x + r.y * r.y + r.z * r.z, bb.x * bb.x + bb.y * bb.y + bb.z * bb.z};
        tile_partial<2>(v, P.tp, P.tiles, t);
    }
}

__global__ void __launch_bounds__(kThreads) k_pool_init(IterArgs<float> a, PoolArgs P, const double* __restrict__ src) {
    const size_t n = a.n;
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        const SlotState& S = P.st[P.tile_scene[t]];
        if (!(S.enabled && S.inner_on)) continue;
        const double scale = S.r64_norm > 0.0 ? 1.0 / S.r64_norm : 1.0;
        const uint32_t i = t * kThreads + threadIdx.x;
        V3<float> r = {(float)(src[i] * scale), (float)(src[n + i] * scale), (float)(src[2 * n + i] * scale)};
        V3<float> z = mul(load_sym(a.Dinv, n, i), r);
        store_v(a.r, n, i, r);
        store_v(a.z, n, i, z);
        store_v(a.x, n, i, V3<float>{0.f, 0.f, 0.f});
        store_v(const_cast<float*>(a.p_old), n, i, V3<float>{0.f, 0.f, 0.f});
        double v[2] = {dot_d(r, z), dot_d(r, r)};
        tile_partial<2>(v, P.tp + P.tiles, P.tiles, t);
    }
}

template <int PAR>
__global__ void __launch_bounds__(kThreads) k_pool_matvec(IterArgs<float> a, PoolArgs P) {
    const size_t n = a.n;
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        const SlotState& S = P.st[P.tile_scene[t]];
        if (!slot_iterating(S)) continue;
        const float beta = (float)S.beta;
        const float* __restrict__ z_in = a.z_in;
        const float* __restrict__ p_old = a.p_old;
        auto get = [&](uint32_t j) {
            return V3<float>{fmaf(beta, __ldg(p_old + j), __ldg(z_in + j)),
                             fmaf(beta, __ldg(p_old + n + j), __ldg(z_in + n + j)),
                             fmaf(beta, __ldg(p_old + 2 * n + j), __ldg(z_in + 2 * n + j))};
        };
        const uint32_t i = t * kThreads + threadIdx.x;
        V3<float> pi = get(i);
        V3<float> y = apply_row<float>(a, i, pi, get);
        store_v(a.p_new, n, i, pi);
        store_v(a.ap, n, i, y);
        double v[1] = {dot_d(pi, y)};
        tile_partial<1>(v, P.tp, P.tiles, t);
    }
}

__global__ void __launch_bounds__(kThreads) k_pool_update(IterArgs<float> a, PoolArgs P) {
    const size_t n = a.n;
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        const SlotState& S = P.st[P.tile_scene[t]];
        if (!slot_iterating(S)) continue;
        const float alpha = (float)S.alpha;
        const uint32_t i = t * kThreads + threadIdx.x;
        V3<float> p = ldg_v(a.p_new, n, i);
        V3<float> ap = ldg_v(a.ap, n, i);
        V3<float> x = load_v(a.x, n, i);
        V3<float> r = load_v(a.r, n, i);
        Sym<float> M = load_sym(a.Dinv, n, i);
        x = {fmaf(alpha, p.x, x.x), fmaf(alpha, p.y, x.y), fmaf(alpha, p.z, x.z)};
        r = {fmaf(-alpha, ap.x, r.x), fmaf(-alpha, ap.y, r.y), fmaf(-alpha, ap.z, r.z)};
        V3<float> z = mul(M, r);
        store_v(a.x, n, i, x);
        store_v(a.r, n, i, r);
        store_v(a.z, n, i, z);
        double v[2] = {dot_d(r, z), dot_d(r, r)};
        tile_partial<2>(v, P.tp + P.tiles, P.tiles, t);
    }
}

__global__ void __launch_bounds__(kThreads) k_pool_accumulate(PoolArgs P, double* __restrict__ x64,
                                                              const float* __restrict__ x32, uint32_t n) {
    for (uint32_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        if (!P.tile_on[t]) continue;
        const SlotState& S = P.st[P.tile_scene[t]];
        if (!(S.enabled && S.inner_on)) continue;
        const size_t i = (size_t)t * kThreads + threadIdx.x;
#pragma unroll
        for (int c = 0; c < 3; ++c) x64[c * (size_t)n + i] += S.r64_norm * (double)x32[c * (size_t)n + i];
    }
}

// ---- per-slot kernels (one warp per slot) --------------------------------------------
__device__ __forceinline__ int32_t slot_of_warp(const PoolArgs& P) {
    uint32_t s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    return s < P.slots ? (int32_t)s : -1;
}

// Outer refinement step: book the last inner solve, then test |b - A x| / |b|.
__global__ void k_pool_outer(PoolArgs P) {
    const int32_t s = slot_of_warp(P);
    if (s < 0) return;
    SlotState& S = P.st[s];
    if (!S.enabled || S.outer_done) return;
    const bool lane0 = (threadIdx.x & 31) == 0;
    const double rr = warp_total(P.tp, P.slot_first[s], P.slot_tiles[s]);
    const double bb = warp_total(P.tp + P.tiles, P.slot_first[s], P.slot_tiles[s]);
    if (!lane0) return;
    if (S.inner_on) {
        S.used += S.its;
        S.outer += 1;
        S.inner_on = 0;
        if (S.status_in == VX_NONFINITE) {
            S.outer_done = 1;
            S.status = VX_NONFINITE;
            return;
        }
    }
    S.r64_norm = sqrt(rr);
    S.b_norm = sqrt(bb);
    S.residual = S.b_norm > 0.0 ? S.r64_norm / S.b_norm : 0.0;
    if (!isfinite(S.residual)) {
        S.outer_done = 1;
        S.status = VX_NONFINITE;
    } else if (S.b_norm <= 1e-12 || S.residual <= P.tolerance) {
        S.outer_done = 1;
        S.status = VX_OK;
    } else if (S.used >= P.max_iterations || S.outer >= P.max_outer) {
        S.outer_done = 1;
        S.status = VX_NOT_CONVERGED;
    } else {
        S.inner_on = 1;
        S.tol_in = fmax(P.inner_tolerance, 0.5 * P.tolerance / S.residual);
        S.max_its = P.max_iterations - S.used;
        atomicAdd(P.pending, 1);
    }
}

__global__ void k_pool_scal_init(PoolArgs P) {
    const int32_t s = slot_of_warp(P);
    if (s < 0) return;
    SlotState& S = P.st[s];
    if (!(S.enabled && S.inner_on)) return;
    const double rz = warp_total(P.tp + P.tiles, P.slot_first[s], P.slot_tiles[s]);
    const double rr = warp_total(P.tp + 2 * (size_t)P.tiles, P.slot_first[s], P.slot_tiles[s]);
    if ((threadIdx.x & 31) != 0) return;
    S.rz = rz;
    S.initial = sqrt(rr);
    S.its = 0;
    S.beta = 0.0;
    S.alpha = 0.0;
    S.residual_in = 0.0;
    S.status_in = VX_OK;
    S.done = 0;
    if (!isfinite(rr) || !isfinite(rz)) {
        S.done = 1;
        S.status_in = VX_NONFINITE;
    } else if (!(S.initial > 1e-12)) {
        S.done = 1;
    } else if (S.max_its == 0) {
        S.done = 1;
        S.status_in = VX_NOT_CONVERGED;
    }
    if (!S.done) atomicAdd(P.active, 1);
}

__global__ void k_pool_alpha(PoolArgs P) {
    const int32_t s = slot_of_warp(P);
    if (s < 0) return;
    SlotState& S = P.st[s];
    if (!slot_iterating(S)) return;
    const double pap = warp_total(P.tp, P.slot_first[s], P.slot_tiles[s]);
    if ((threadIdx.x & 31) != 0) return;
    if (!isfinite(pap) || pap <= 1e-30) {
        S.its += 1;  // the matvec happened (src/solver.rs:1861-1866)
        if (!isfinite(pap)) S.status_in = VX_NONFINITE;
        S.done = 1;
        atomicSub(P.active, 1);
        return;
    }
    S.alpha = (double)(float)(S.rz / pap);
}

__global__ void k_pool_beta(PoolArgs P) {
    const int32_t s = slot_of_warp(P);
    if (s < 0) return;
    SlotState& S = P.st[s];
    if (!slot_iterating(S)) return;
    const double rz = warp_total(P.tp + P.tiles, P.slot_first[s], P.slot_tiles[s]);
    const double rr = warp_total(P.tp + 2 * (size_t)P.tiles, P.slot_first[s], P.slot_tiles[s]);
    if ((threadIdx.x & 31) != 0) return;
    S.its += 1;
    const double residual = sqrt(rr) / S.initial;
    S.residual_in = residual;
    int32_t stop = 1;
    if (!isfinite(rr) || !isfinite(rz)) {
        S.status_in = VX_NONFINITE;
    } else if (residual < S.tol_in) {
        S.status_in = VX_OK;
    } else if (S.its >= S.max_its) {
        S.status_in = VX_NOT_CONVERGED;
    } else {
        stop = 0;
        S.beta = (double)(float)(rz / S.rz);
        S.rz = rz;
    }
    if (stop) {
        S.done = 1;
        atomicSub(P.active, 1);
    }
}

// ---- host side -------------------------------------------------------------------------
PoolArgs pool_args(vx_pool* p, const vx_pass_params* prm) {
    PoolArgs P;
    P.tiles = p->tiles;
    P.slots = p->slots;
    P.tile_on = p->s.tile_on;
    P.tile_scene = p->s.tile_scene;
    P.slot_first = p->slot_first;
    P.slot_tiles = p->slot_tiles;
    P.st = p->st;
    P.tp = p->s.partials;
    P.active = p->active;
    P.pending = p->pending;
    P.tolerance = prm ? prm->tolerance : 0.0;
    P.inner_tolerance = prm && prm->inner_tolerance > 0.0 ? prm->inner_tolerance : 1e-5;
    P.max_iterations = prm ? prm->max_iterations : 0;
    P.max_outer = prm && prm->max_outer ? prm->max_outer : 30;
    return P;
}

IterArgs<float> pool_args32(vx_scene* s, int ping) {
    IterArgs<float> a{};
    a.n = s->n;
    a.kn = kstride32(s->n);
    a.flags = s->flags;
    a.D = s->d32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.nbr = s->nbr;
    a.rev = s->rev;
    a.mh2 = s->mh2_32;
    a.z_in = s->z32;
    a.p_old = s->p32[ping];
    a.p_new = s->p32[ping ^ 1];
    a.ap = s->ap32;
    a.x = s->x32;
    a.r = s->r32;
    a.z = s->z32;
    return a;
}

IterArgs<double> pool_args64(vx_scene* s) {
    IterArgs<double> a{};
    a.n = s->n;
    a.kn = s->n;
    a.flags = s->flags;
    a.D = s->d64;
    a.K = s->bonds.k64;
    a.Dinv = s->dinv64;
    a.nbr = s->nbr;
    a.rev = s->rev;
    a.x = s->x64;
    return a;
}

unsigned pool_grid(vx_pool* p) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pool_matvec<0>, kThreads, 0);
    if (occ < 1) occ = 1;
    unsigned g = (unsigned)(p->s.sm_count * occ);
    return g < p->tiles ? g : p->tiles;
}

unsigned slot_grid(vx_pool* p) { return (p->slots + 7) / 8; }

cudaError_t pool_chunk_graph(vx_pool* p, const PoolArgs& P) {
    if (p->chunk) return cudaSuccess;
    vx_scene* s = &p->s;
    const unsigned G = pool_grid(p), GS = slot_grid(p);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    for (int it = 0; it < kPoolChunk; it += 2) {
        IterArgs<float> a0 = pool_args32(s, 0), a1 = pool_args32(s, 1);
        k_pool_matvec<0><<<G, kThreads, 0, s->stream>>>(a0, P);
        k_pool_alpha<<<GS, 256, 0, s->stream>>>(P);
        k_pool_update<<<G, kThreads, 0, s->stream>>>(a0, P);
        k_pool_beta<<<GS, 256, 0, s->stream>>>(P);
        k_pool_matvec<1><<<G, kThreads, 0, s->stream>>>(a1, P);
        k_pool_alpha<<<GS, 256, 0, s->stream>>>(P);
        k_pool_update<<<G, kThreads, 0, s->stream>>>(a1, P);
        k_pool_beta<<<GS, 256, 0, s->stream>>>(P);
    }
    e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&p->chunk, g, 0);
    cudaGraphDestroy(g);
    return e;
}

#define VX_POOL_TRY(expr, what)                                                   \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) {                                                  \
            set_error("%s failed: %s", what, cudaGetErrorString(_e));             \
            return _e == cudaErrorMemoryAllocation ? VX_OOM : VX_CUDA_ERROR;      \
        }                                                                         \
    } while (0)

// Marks the tiles of the selected occupied slots.
int32_t pool_select(vx_pool* p, const uint8_t* enabled, std::vector<uint8_t>& on_slot) {
    on_slot.assign(p->slots, 0);
    for (uint32_t k = 0; k < p->slots; ++k) on_slot[k] = p->used[k] && (!enabled || enabled[k]);
    for (uint32_t t = 0; t < p->tiles; ++t)
        p->h_tile_on[t] = p->owner[t] != VX_EMPTY_U32 && on_slot[p->owner[t]] ? 1 : 0;
    VX_POOL_TRY(cudaMemcpyAsync(p->s.tile_on, p->h_tile_on.data(), p->tiles, cudaMemcpyHostToDevice, p->s.stream),
                "pool tile mask");
    return VX_OK;
}

// Packs the occupied slots into waves of the persistent inner solve: a slot of
// n REVs takes ceil(n / 1,536) blocks of equal size, slots go largest first to
// the first wave with room (at most one block per SM), and each wave is one
// cooperative launch. A slot's blocks and sums depend on its own size only, so
// its iterates do not depend on which slots share its wave. The waves are
// unavailable when the device has no cooperative launch or a neighbour delta
// of the pool does not fit the kernel's 16-bit table.
bool pool_waves(vx_pool* p) {
    vx_scene* s = &p->s;
    if (s->nbcode_state == 0) {  // once per topology (launch_reverse_neighbors resets it)
        uint32_t bad = 0;
        if (cudaMemcpyAsync(&bad, s->nbcode_bad, sizeof bad, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            return false;
        s->nbcode_state = bad == 0 ? 1 : 2;
    }
    if (s->nbcode_state != 1) return false;
    if (!p->waves_dirty) return p->waves_ok;
    p->waves_dirty = false;
    p->waves_ok = false;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, s->device);
    if (!coop) return false;
    const uint32_t cap_max = persistent_block_cap();
    const unsigned G_max = (unsigned)s->sm_count;
    std::vector<uint32_t> order;
    for (uint32_t k = 0; k < p->slots; ++k)
        if (p->used[k] && p->rev_n[k]) order.push_back(k);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return p->rev_n[a] > p->rev_n[b]; });
    struct Wave {
        unsigned blocks = 0;
        std::vector<uint32_t> slots;
    };
    std::vector<Wave> ws;
    for (uint32_t k : order) {
        const unsigned nb = (p->rev_n[k] + cap_max - 1) / cap_max;
        if (nb > G_max || nb > 0xFFFFu) return false;
        size_t w = 0;
        while (w < ws.size() && ws[w].blocks + nb > G_max) ++w;
        if (w == ws.size()) ws.emplace_back();
        ws[w].blocks += nb;
        ws[w].slots.push_back(k);
    }
    p->wave_rows.clear();
    p->waves.clear();
    for (const Wave& w : ws) {
        const uint32_t first_row = (uint32_t)p->wave_rows.size();
        uint32_t largest = 0, fb = 0;
        for (uint32_t k : w.slots) {
            const uint32_t n = p->rev_n[k], nb = (n + cap_max - 1) / cap_max, cap = (n + nb - 1) / nb;
            const uint32_t base = p->first[k] * 256u;
            for (uint32_t b = 0; b < nb; ++b) {
                const uint32_t lo = b * cap, cnt = std::min(cap, n - lo);
                p->wave_rows.push_back(make_uint4(base + lo, cnt, k, (fb << 16) | nb));
                largest = std::max(largest, cnt);
            }
            fb += nb;
        }
        p->waves.push_back(make_uint4(first_row, w.blocks, largest, 0));
    }
    if (p->d_wave_rows) {
        cudaStreamSynchronize(s->stream);
        cudaFree(p->d_wave_rows);
        p->d_wave_rows = nullptr;
    }
    if (p->wave_rows.empty()) return false;
    if (cudaMalloc(&p->d_wave_rows, p->wave_rows.size() * sizeof(uint4)) != cudaSuccess) {
        (void)cudaGetLastError();
        p->d_wave_rows = nullptr;
        return false;
    }
    if (cudaMemcpy(p->d_wave_rows, p->wave_rows.data(), p->wave_rows.size() * sizeof(uint4), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return false;
    p->waves_ok = true;
    return true;
}

int32_t pool_solve(vx_pool* p, const vx_pass_params* prm, const std::vector<uint8_t>& on_slot, vx_pass_stats* out) {
    vx_scene* s = &p->s;
    cudaStream_t st = s->stream;
    PoolArgs P = pool_args(p, prm);
    const unsigned G = pool_grid(p), GS = slot_grid(p);
    for (uint32_t k = 0; k < p->slots; ++k) {
        std::memset(&p->h_st[k], 0, sizeof(SlotState));
        p->h_st[k].enabled = on_slot[k];
        p->h_st[k].status = VX_NOT_CONVERGED;
    }
    VX_POOL_TRY(cudaMemcpyAsync(p->st, p->h_st, p->slots * sizeof(SlotState), cudaMemcpyHostToDevice, st), "pool state");
    k_pool_zero<<<G, kThreads, 0, st>>>(P, s->x64, s->n);
    // the inner solves: persistent waves (VX_KERNEL_PERSISTENT) or the chunk
    // graph of tile kernels (VX_KERNEL_AUTO / STREAMING). The waves run one after
    // another, each as long as its slowest slot, where the tile kernels advance
    // every slot at once; on the batched workload the tile kernels measured
    // faster, so they are the default.
    const bool waves = prm->kernel == VX_KERNEL_PERSISTENT && pool_waves(p);
    if (prm->kernel == VX_KERNEL_PERSISTENT && !waves) {
        set_error("vx_pool_pass: the persistent inner solve is not available for this pool");
        return VX_BAD_INPUT;
    }
    if (!waves) VX_POOL_TRY(pool_chunk_graph(p, P), "pool graph capture");
    IterArgs<double> a64 = pool_args64(s);
    const uint32_t outer_cap = P.max_outer + 2;
    for (uint32_t outer = 0; outer < outer_cap; ++outer) {
        VX_POOL_TRY(cudaMemsetAsync(p->pending, 0, sizeof(int32_t), st), "pool");
        k_pool_residual64<<<G, kThreads, 0, st>>>(a64, P, s->b64, s->r64);
        k_pool_outer<<<GS, 256, 0, st>>>(P);
        s->launches += 2;
        VX_POOL_TRY(cudaMemcpyAsync(&p->h_flag[0], p->pending, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "pool");
        VX_POOL_TRY(cudaStreamSynchronize(st), "pool outer step");
        if (p->h_flag[0] == 0) break;
        if (waves) {
            // the one-reduction form (vx_expanded.cu); VXCOROT_PERSISTENT=range
            // keeps the classic two-reduction form of vx_persistent.cu
            const char* form = std::getenv("VXCOROT_PERSISTENT");
            const bool classic = form && std::strcmp(form, "range") == 0;
            for (const uint4& w : p->waves) {
                int32_t r = classic ? solve_inner_slots(s, p->d_wave_rows + w.x, p->st, w.y, w.z)
                                    : solve_inner_slots_expanded(s, p->d_wave_rows + w.x, p->st, w.y, w.z);
                if (r != VX_OK) return r;
            }
            VX_POOL_TRY(cudaMemcpyAsync(&p->h_flag[3], s->barrier + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
                        "pool");
            VX_POOL_TRY(cudaStreamSynchronize(st), "pool inner solve");
            if (p->h_flag[3]) {
                set_error("persistent pool PCG: a grid barrier wait ran out");
                return VX_TIMEOUT;
            }
            k_pool_accumulate<<<G, kThreads, 0, st>>>(P, s->x64, s->x32, s->n);
            s->launches += 1;
            continue;
        }
        VX_POOL_TRY(cudaMemsetAsync(p->active, 0, sizeof(int32_t), st), "pool");
        k_pool_init<<<G, kThreads, 0, st>>>(pool_args32(s, 0), P, s->r64);
        k_pool_scal_init<<<GS, 256, 0, st>>>(P);
        s->launches += 2;
        const uint32_t chunks = P.max_iterations / kPoolChunk + 2;
        bool seen_done = false;
        for (uint32_t c = 0; c < chunks && !seen_done; ++c) {
            VX_POOL_TRY(cudaGraphLaunch(p->chunk, st), "pool chunk");
            s->launches += 4 * kPoolChunk;
            VX_POOL_TRY(cudaMemcpyAsync(&p->h_flag[1 + (c & 1)], p->active, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
                        "pool");
            VX_POOL_TRY(cudaEventRecord(s->ev[c & 1], st), "pool");
            if (c >= 1) {
                VX_POOL_TRY(cudaEventSynchronize(s->ev[(c - 1) & 1]), "pool chunk");
                seen_done = p->h_flag[1 + ((c - 1) & 1)] == 0;
            }
        }
        k_pool_accumulate<<<G, kThreads, 0, st>>>(P, s->x64, s->x32, s->n);
        s->launches += 1;
    }
    VX_POOL_TRY(cudaMemcpyAsync(p->h_st, p->st, p->slots * sizeof(SlotState), cudaMemcpyDeviceToHost, st), "pool state");
    VX_POOL_TRY(cudaStreamSynchronize(st), "pool solve");
    int32_t worst = VX_OK;
    for (uint32_t k = 0; k < p->slots; ++k) {
        if (!on_slot[k]) continue;
        const SlotState& S = p->h_st[k];
        int32_t status = S.outer_done ? S.status : VX_NOT_CONVERGED;
        if (out) {
            out[k].iterations = S.used;
            out[k].outer_iterations = S.outer;
            out[k].residual = S.residual;
            out[k].true_residual = S.residual;
            out[k].converged = status == VX_OK;
            out[k].active = p->rev_n[k];
        }
        if (status == VX_NONFINITE) worst = VX_NONFINITE;
        else if (status != VX_OK && worst == VX_OK) worst = status;
    }
    return worst;
}

}  // namespace
}  // namespace vx

using namespace vx;

namespace vx {
// Replaces an idle pool's stream by one of the given priority (lower numbers
// run first when the GPU is shared). Only before the pool captures graphs.
int32_t pool_stream_priority(vx_pool* p, int priority) {
    cudaSetDevice(p->s.device);
    cudaStream_t fresh = nullptr;
    cudaError_t e = cudaStreamSynchronize(p->s.stream);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&fresh, cudaStreamNonBlocking, priority);
    if (e != cudaSuccess) {
        set_error("pool stream priority: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    cudaStreamDestroy(p->s.stream);
    p->s.stream = fresh;
    return VX_OK;
}
}  // namespace vx

extern "C" {

uint64_t vx_pool_footprint_bytes(uint64_t max_revs, uint32_t max_slots) {
    uint64_t cap = (max_revs + 255) / 256 * 256;
    if (cap > 0x7FFFFF00ull) return 0;
    uint64_t tiles = cap / 256;
    return scene_bytes((uint32_t)cap, VX_POOL_MATERIALS * max_slots) + tiles * 5 + max_slots * (sizeof(SlotState) + 16) +
           4096;
}

int32_t vx_pool_create(vx_ctx* ctx, uint64_t max_revs, uint32_t max_slots, vx_pool** out) {
    clear_error();
    if (!ctx || !out || max_revs == 0 || max_slots == 0) {
        set_error("vx_pool_create: bad argument");
        return VX_BAD_INPUT;
    }
    uint64_t cap = (max_revs + 255) / 256 * 256;
    if (cap >= 0x7FFFFFFFull / 3) {
        set_error("vx_pool_create: capacity of %llu REVs exceeds the index range", (unsigned long long)cap);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(ctx->device);
    vx_pool* p = new (std::nothrow) vx_pool();
    if (!p) return VX_OOM;
    if ((size_t)max_slots * 3 > 4 * kPoolStageRevs) {
        set_error("vx_pool_create: %u slots exceed the staging of per-slot scalars", max_slots);
        delete p;
        return VX_BAD_INPUT;
    }
    int32_t r = scene_alloc(&p->s, ctx, (uint32_t)cap, VX_POOL_MATERIALS * max_slots, kPoolStageRevs);
    if (r != VX_OK) {
        delete p;
        return r;
    }
    p->slots = max_slots;
    p->tiles = (uint32_t)(cap / 256);
    p->owner.assign(p->tiles, VX_EMPTY_U32);
    p->first.assign(max_slots, 0);
    p->count.assign(max_slots, 0);
    p->rev_n.assign(max_slots, 0);
    p->used.assign(max_slots, 0);
    p->h_tile_on.assign(p->tiles, 0);
    size_t al = 256, off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + al - 1) / al * al;
        return o;
    };
    size_t o_on = take(p->tiles), o_ts = take(p->tiles * 4), o_st = take(max_slots * sizeof(SlotState)),
           o_first = take(max_slots * 4), o_cnt = take(max_slots * 4), o_act = take(16), o_ang = take(max_slots * 8),
           o_revs = take(max_slots * 4);
    cudaError_t e = cudaMalloc(&p->extra, off);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->extra, 0, off, p->s.stream);
    if (e == cudaSuccess) e = cudaMallocHost(&p->h_st, max_slots * sizeof(SlotState));
    if (e == cudaSuccess) e = cudaMallocHost(&p->h_flag, 4 * sizeof(int32_t));
    if (e != cudaSuccess) {
        set_error("vx_pool_create: allocation failed: %s", cudaGetErrorString(e));
        vx_pool_destroy(p);
        return VX_OOM;
    }
    p->s.tile_on = (uint8_t*)(p->extra + o_on);
    p->s.tile_scene = (uint32_t*)(p->extra + o_ts);
    p->st = (SlotState*)(p->extra + o_st);
    p->slot_first = (uint32_t*)(p->extra + o_first);
    p->slot_tiles = (uint32_t*)(p->extra + o_cnt);
    p->slot_revs = (uint32_t*)(p->extra + o_revs);
    p->s.pool_slot_first = p->slot_first;
    p->s.pool_slot_revs = p->slot_revs;
    p->active = (int32_t*)(p->extra + o_act);
    p->pending = p->active + 1;
    p->angle = (unsigned long long*)(p->extra + o_ang);
    p->s.max_angle_bits = p->angle;
    p->s.pool_slots = max_slots;
    // the free arena is inert: no tile is on, every tile maps to no slot, and no
    // REV has a neighbour (a zeroed table would bond every free REV to REV 0
    // and give REV 0 a reverse neighbour picked by whichever write lands last)
    std::vector<uint32_t> ts(p->tiles, VX_EMPTY_U32);
    e = cudaMemcpyAsync(p->s.tile_scene, ts.data(), p->tiles * 4, cudaMemcpyHostToDevice, p->s.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->s.nbr, 0xFF, 3 * (size_t)p->s.n * sizeof(uint32_t), p->s.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->s.rev, 0xFF, 3 * (size_t)p->s.n * sizeof(uint32_t), p->s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->s.stream);
    if (e != cudaSuccess) {
        set_error("vx_pool_create: %s", cudaGetErrorString(e));
        vx_pool_destroy(p);
        return VX_CUDA_ERROR;
    }
    *out = p;
    return VX_OK;
}

int32_t vx_pool_destroy(vx_pool* p) {
    if (!p) return VX_OK;
    cudaSetDevice(p->s.device);
    if (p->s.stream) cudaStreamSynchronize(p->s.stream);
    if (p->chunk) cudaGraphExecDestroy(p->chunk);
    if (p->d_wave_rows) cudaFree(p->d_wave_rows);
    if (p->extra) cudaFree(p->extra);
    if (p->h_st) cudaFreeHost(p->h_st);
    if (p->h_flag) cudaFreeHost(p->h_flag);
    p->s.max_angle_bits = nullptr;
    scene_release(&p->s);
    delete p;
    return VX_OK;
}

uint32_t vx_pool_capacity_slots(vx_pool* p) { return p ? p->slots : 0; }

int32_t vx_pool_free_revs(vx_pool* p, uint64_t* out_free, uint64_t* out_largest) {
    if (!p) return VX_BAD_INPUT;
    uint64_t fr = 0, best = 0, run = 0;
    for (uint32_t t = 0; t < p->tiles; ++t) {
        if (p->owner[t] == VX_EMPTY_U32) {
            ++fr;
            ++run;
            best = std::max(best, run);
        } else {
            run = 0;
        }
    }
    if (out_free) *out_free = fr * 256;
    if (out_largest) *out_largest = best * 256;
    return VX_OK;
}

// Adds a scene to the first tile range that holds it.
int32_t vx_pool_add(vx_pool* p, const vx_scene_desc* d, uint32_t* out_slot) {
    clear_error();
    if (!p || !d || !out_slot) {
        set_error("vx_pool_add: null argument");
        return VX_BAD_INPUT;
    }
    const uint32_t n = d->n;
    if (n == 0 || !d->position || !d->kinematic || !d->mass || !d->material || !d->materials || !d->fiber ||
        !d->anisotropy || !d->neighbor) {
        set_error("vx_pool_add: empty scene or a required array is null");
        return VX_BAD_INPUT;
    }
    if (d->material_count == 0 || d->material_count > VX_POOL_MATERIALS) {
        set_error("vx_pool_add: %u materials; a pooled scene has 1..%d", d->material_count, VX_POOL_MATERIALS);
        return VX_BAD_INPUT;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (d->material[i] >= d->material_count) {
            set_error("vx_pool_add: REV %u has material %u of %u", i, d->material[i], d->material_count);
            return VX_BAD_INPUT;
        }
        for (int c = 0; c < 3; ++c)
            if (!std::isfinite(d->position[3 * (size_t)i + c])) {
                set_error("vx_pool_add: non-finite position of REV %u", i);
                return VX_NONFINITE;
            }
    }
    for (size_t e = 0; e < 3 * (size_t)n; ++e)
        if (d->neighbor[e] != VX_EMPTY && d->neighbor[e] >= n) {
            set_error("vx_pool_add: bond %zu points at REV %u of %u", e, d->neighbor[e], n);
            return VX_BAD_INPUT;
        }
    uint32_t slot = VX_EMPTY_U32;
    for (uint32_t k = 0; k < p->slots; ++k)
        if (!p->used[k]) {
            slot = k;
            break;
        }
    if (slot == VX_EMPTY_U32) {
        set_error("vx_pool_add: all %u slots are occupied", p->slots);
        return VX_OOM;
    }
    const uint32_t need = (n + 255) / 256;
    uint32_t start = VX_EMPTY_U32, run = 0;
    for (uint32_t t = 0; t < p->tiles; ++t) {
        run = p->owner[t] == VX_EMPTY_U32 ? run + 1 : 0;
        if (run == need) {
            start = t + 1 - need;
            break;
        }
    }
    if (start == VX_EMPTY_U32) {
        set_error("vx_pool_add: no free range of %u tiles (%u REVs)", need, n);
        return VX_OOM;
    }
    vx_scene* s = &p->s;
    cudaSetDevice(s->device);
    const size_t C = s->n, base = (size_t)start * 256, m = (size_t)need * 256;
    const uint32_t mat0 = slot * VX_POOL_MATERIALS;
    // host staging of the slot's tile range in the arena layout
    std::vector<double> pos(3 * m, 0.0);
    std::vector<double4> rot(m, make_double4(0.0, 0.0, 0.0, 1.0));
    std::vector<uint8_t> kin(m, 1);
    std::vector<uint32_t> mat(m, mat0), nbr(3 * m, VX_EMPTY);
    std::vector<float4> p0(m, make_float4(0.f, 0.f, 1.f, 0.f)), p1(m, make_float4(1.f, 1.f, 0.f, 1.f)), ba(3 * m),
        bb(3 * m);
    for (size_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) pos[c * m + i] = d->position[3 * i + c];
        if (d->rotation)
            rot[i] = make_double4(d->rotation[4 * i], d->rotation[4 * i + 1], d->rotation[4 * i + 2], d->rotation[4 * i + 3]);
        kin[i] = d->kinematic[i];
        mat[i] = mat0 + d->material[i];
        p0[i] = make_float4(d->fiber[3 * i], d->fiber[3 * i + 1], d->fiber[3 * i + 2], d->anisotropy[i]);
        p1[i] = make_float4(d->solid_fraction ? d->solid_fraction[i] : 1.0f,
                            d->thermal_strength ? d->thermal_strength[i] : 1.0f,
                            d->thermal_delta ? d->thermal_delta[i] : 0.0f, d->mass[i]);
    }
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < n; ++i) {
            size_t e = (size_t)a * n + i;
            uint32_t j = d->neighbor[e];
            nbr[a * m + i] = j == VX_EMPTY ? VX_EMPTY : (uint32_t)(base + j);
            float fo[3] = {0, 0, 0}, pl[3] = {0, 0, 0};
            if (d->formation_offset)
                for (int c = 0; c < 3; ++c) fo[c] = d->formation_offset[3 * e + c];
            if (d->plastic_strain)
                for (int c = 0; c < 3; ++c) pl[c] = d->plastic_strain[3 * e + c];
            ba[a * m + i] = make_float4(fo[0], fo[1], fo[2], d->damage ? d->damage[e] : 0.0f);
            bb[a * m + i] = make_float4(pl[0], pl[1], pl[2], 0.0f);
        }
    cudaStream_t st = s->stream;
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
        e = cudaMemcpyAsync(s->pos + c * C + base, pos.data() + c * m, m * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->pred + c * C + base, pos.data() + c * m, m * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->loads + c * C + base, 0, m * 8, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->vel + c * C + base, 0, m * 8, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->bond_c + c * C + base, 0, m * sizeof(float4), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->bond_d + c * C + base, 0, m * sizeof(float), st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->nbr + c * C + base, nbr.data() + c * m, m * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->bond_a + c * C + base, ba.data() + c * m, m * sizeof(float4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->bond_b + c * C + base, bb.data() + c * m, m * sizeof(float4), cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->rot + base, rot.data(), m * sizeof(double4), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->kin + base, kin.data(), m, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->tmask + base, 0, m, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->matid + base, mat.data(), m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->param0 + base, p0.data(), m * sizeof(float4), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->param1 + base, p1.data(), m * sizeof(float4), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->materials + mat0, d->materials, d->material_count * sizeof(vx_material),
                            cudaMemcpyHostToDevice, st);
    std::vector<uint32_t> ts(need, slot);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->tile_scene + start, ts.data(), need * 4, cudaMemcpyHostToDevice, st);
    uint32_t fc[3] = {start, need, (uint32_t)n};
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->slot_first + slot, &fc[0], 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->slot_tiles + slot, &fc[1], 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->slot_revs + slot, &fc[2], 4, cudaMemcpyHostToDevice, st);
    for (int c = 0; c < 3 && e == cudaSuccess; ++c)
        e = cudaMemcpyAsync(s->prev + c * C + base, pos.data() + c * m, m * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_rest_range(s, base, m);
    if (e == cudaSuccess) e = launch_reverse_neighbors(s);
    if (e == cudaSuccess) e = launch_flags(s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error("vx_pool_add: upload failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    for (uint32_t t = start; t < start + need; ++t) p->owner[t] = slot;
    p->first[slot] = start;
    p->count[slot] = need;
    p->rev_n[slot] = n;
    p->used[slot] = 1;
    p->waves_dirty = true;
    *out_slot = slot;
    return VX_OK;
}

int32_t vx_pool_remove(vx_pool* p, uint32_t slot) {
    clear_error();
    if (!p || slot >= p->slots || !p->used[slot]) {
        set_error("vx_pool_remove: no scene in slot %u", slot);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    std::vector<uint32_t> ts(p->count[slot], VX_EMPTY_U32);
    cudaError_t e = cudaMemcpyAsync(p->s.tile_scene + p->first[slot], ts.data(), ts.size() * 4, cudaMemcpyHostToDevice,
                                    p->s.stream);
    // the freed tiles lose their bonds again, and the reverse table forgets them
    const size_t base = (size_t)p->first[slot] * 256, m = (size_t)p->count[slot] * 256, C = p->s.n;
    for (int a = 0; a < 3 && e == cudaSuccess; ++a)
        e = cudaMemsetAsync(p->s.nbr + a * C + base, 0xFF, m * sizeof(uint32_t), p->s.stream);
    if (e == cudaSuccess) e = launch_reverse_neighbors(&p->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->s.stream);
    if (e != cudaSuccess) {
        set_error("vx_pool_remove: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    for (uint32_t t = p->first[slot]; t < p->first[slot] + p->count[slot]; ++t) p->owner[t] = VX_EMPTY_U32;
    p->used[slot] = 0;
    p->rev_n[slot] = 0;
    p->waves_dirty = true;
    return VX_OK;
}

static int32_t slot_ok(vx_pool* p, uint32_t slot, const void* ptr, const char* fn) {
    clear_error();
    if (!p || slot >= p->slots || !p->used[slot] || !ptr) {
        set_error("%s: no scene in slot %u or null argument", fn, slot);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    return VX_OK;
}

// per-slot vector copies: AoS host <-> SoA arena range
static int32_t slot_vec(vx_pool* p, uint32_t slot, double* dev, double* host, bool upload) {
    vx_scene* s = &p->s;
    const size_t C = s->n, base = (size_t)p->first[slot] * 256, n = p->rev_n[slot];
    double* stage = s->h_stage;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    // chunks of at most stage_revs REVs (AoS host <-> SoA device)
    for (size_t lo = 0; lo < n && e == cudaSuccess; lo += s->stage_revs) {
        const size_t m = std::min(s->stage_revs, n - lo);
        if (upload) {
            for (size_t i = 0; i < m; ++i)
                for (int c = 0; c < 3; ++c) stage[c * m + i] = host[3 * (lo + i) + c];
            for (int c = 0; c < 3 && e == cudaSuccess; ++c)
                e = cudaMemcpyAsync(dev + c * C + base + lo, stage + c * m, m * 8, cudaMemcpyHostToDevice, s->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        } else {
            for (int c = 0; c < 3 && e == cudaSuccess; ++c)
                e = cudaMemcpyAsync(stage + c * m, dev + c * C + base + lo, m * 8, cudaMemcpyDeviceToHost, s->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            if (e == cudaSuccess)
                for (size_t i = 0; i < m; ++i)
                    for (int c = 0; c < 3; ++c) host[3 * (lo + i) + c] = stage[c * m + i];
        }
    }
    if (e != cudaSuccess) {
        set_error("pool copy failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

int32_t vx_pool_set_positions(vx_pool* p, uint32_t slot, const double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    for (size_t t = 0; t < 3 * (size_t)p->rev_n[slot]; ++t)
        if (!std::isfinite(xyz[t])) {
            set_error("vx_pool_set_positions: non-finite value at %zu", t);
            return VX_NONFINITE;
        }
    return slot_vec(p, slot, p->s.pos, const_cast<double*>(xyz), true);
}
int32_t vx_pool_set_previous(vx_pool* p, uint32_t slot, const double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    for (size_t t = 0; t < 3 * (size_t)p->rev_n[slot]; ++t)
        if (!std::isfinite(xyz[t])) {
            set_error("vx_pool_set_previous: non-finite value at %zu", t);
            return VX_NONFINITE;
        }
    return slot_vec(p, slot, p->s.prev, const_cast<double*>(xyz), true);
}
int32_t vx_pool_get_previous(vx_pool* p, uint32_t slot, double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    return slot_vec(p, slot, p->s.prev, xyz, false);
}
int32_t vx_pool_contact_project(vx_pool* p, const uint8_t* enabled, vx_contact_stats* out, uint32_t* slot_contacts) {
    clear_error();
    if (!p) {
        set_error("vx_pool_contact_project: null pool");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    std::vector<uint8_t> sel;
    int32_t r = pool_select(p, enabled, sel);
    if (r != VX_OK) return r;
    return contact_project(&p->s, out, slot_contacts);
}
int32_t vx_pool_get_positions(vx_pool* p, uint32_t slot, double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    return slot_vec(p, slot, p->s.pos, xyz, false);
}
int32_t vx_pool_set_velocities(vx_pool* p, uint32_t slot, const double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    for (size_t t = 0; t < 3 * (size_t)p->rev_n[slot]; ++t)
        if (!std::isfinite(xyz[t])) {
            set_error("vx_pool_set_velocities: non-finite value at %zu", t);
            return VX_NONFINITE;
        }
    return slot_vec(p, slot, p->s.vel, const_cast<double*>(xyz), true);
}
int32_t vx_pool_get_velocities(vx_pool* p, uint32_t slot, double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    return slot_vec(p, slot, p->s.vel, xyz, false);
}
int32_t vx_pool_set_loads(vx_pool* p, uint32_t slot, const double* xyz) {
    int32_t r = slot_ok(p, slot, xyz, __func__);
    if (r != VX_OK) return r;
    return slot_vec(p, slot, p->s.loads, const_cast<double*>(xyz), true);
}
int32_t vx_pool_set_predicted(vx_pool* p, uint32_t slot, const double* xyz) {
    clear_error();
    if (!p || slot >= p->slots || !p->used[slot]) return VX_BAD_INPUT;
    cudaSetDevice(p->s.device);
    if (!xyz) {
        const size_t C = p->s.n, base = (size_t)p->first[slot] * 256, n = p->rev_n[slot];
        for (int c = 0; c < 3; ++c)
            VX_POOL_TRY(cudaMemcpyAsync(p->s.pred + c * C + base, p->s.pos + c * C + base, n * 8, cudaMemcpyDeviceToDevice,
                                        p->s.stream), "predicted");
        VX_POOL_TRY(cudaStreamSynchronize(p->s.stream), "predicted");
        return VX_OK;
    }
    return slot_vec(p, slot, p->s.pred, const_cast<double*>(xyz), true);
}
int32_t vx_pool_set_targets(vx_pool* p, uint32_t slot, const uint8_t* mask, const double* xyz) {
    int32_t r = slot_ok(p, slot, mask, __func__);
    if (r != VX_OK) return r;
    const size_t base = (size_t)p->first[slot] * 256, n = p->rev_n[slot];
    VX_POOL_TRY(cudaMemcpyAsync(p->s.tmask + base, mask, n, cudaMemcpyHostToDevice, p->s.stream), "targets");
    if (xyz) {
        r = slot_vec(p, slot, p->s.target, const_cast<double*>(xyz), true);
        if (r != VX_OK) return r;
    }
    VX_POOL_TRY(launch_flags(&p->s), "flags");
    VX_POOL_TRY(cudaStreamSynchronize(p->s.stream), "targets");
    return VX_OK;
}
int32_t vx_pool_get_rotations(vx_pool* p, uint32_t slot, double* q) {
    int32_t r = slot_ok(p, slot, q, __func__);
    if (r != VX_OK) return r;
    const size_t base = (size_t)p->first[slot] * 256, n = p->rev_n[slot];
    VX_POOL_TRY(cudaMemcpyAsync(q, p->s.rot + base, n * sizeof(double4), cudaMemcpyDeviceToHost, p->s.stream), "rotations");
    VX_POOL_TRY(cudaStreamSynchronize(p->s.stream), "rotations");
    return VX_OK;
}
int32_t vx_pool_checkpoint(vx_pool* p, int32_t op) { return p ? vx_scene_checkpoint(&p->s, op) : VX_BAD_INPUT; }
void* vx_pool_stream(vx_pool* p) { return p ? (void*)p->s.stream : nullptr; }

int32_t vx_pool_fit_rotations(vx_pool* p, const uint8_t* enabled, double* out_max_angle) {
    clear_error();
    if (!p) return VX_BAD_INPUT;
    cudaSetDevice(p->s.device);
    std::vector<uint8_t> on;
    int32_t r = pool_select(p, enabled, on);
    if (r != VX_OK) return r;
    VX_POOL_TRY(launch_fit_rotations(&p->s), "pool fit_rotations");
    std::vector<unsigned long long> bits(p->slots, 0);
    VX_POOL_TRY(cudaMemcpyAsync(bits.data(), p->angle, p->slots * 8, cudaMemcpyDeviceToHost, p->s.stream), "angles");
    VX_POOL_TRY(cudaStreamSynchronize(p->s.stream), "pool fit_rotations");
    if (out_max_angle)
        for (uint32_t k = 0; k < p->slots; ++k) {
            double v;
            std::memcpy(&v, &bits[k], 8);
            out_max_angle[k] = on[k] ? v : 0.0;
        }
    return VX_OK;
}

int32_t vx_pool_pass(vx_pool* p, const uint8_t* enabled, const vx_pass_params* prm, vx_pass_stats* out) {
    clear_error();
    if (!p || !prm) {
        set_error("vx_pool_pass: null argument");
        return VX_BAD_INPUT;
    }
    if (!(prm->h > 0.0) || !std::isfinite(prm->h) || !(prm->tolerance > 0.0)) {
        set_error("vx_pool_pass: invalid h=%g or tolerance=%g", prm->h, prm->tolerance);
        return VX_BAD_INPUT;
    }
    if (prm->precision != VX_PRECISION_MIXED) {
        set_error("vx_pool_pass: pools solve the FP32-inner / FP64-refinement form (VX_PRECISION_MIXED)");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    if (out) std::memset(out, 0, p->slots * sizeof(vx_pass_stats));
    std::vector<uint8_t> on;
    int32_t r = pool_select(p, enabled, on);
    if (r != VX_OK) return r;
    vx_scene* s = &p->s;
    s->launches = 2;
    bool reuse = prm->reuse_preconditioner && s->have_dinv;
    VX_POOL_TRY(launch_assembly(s, prm->h, reuse), "pool assembly");
    s->have_dinv = true;
    s->assembled = true;
    int32_t status = pool_solve(p, prm, on, out);
    if (status == VX_CUDA_ERROR || status == VX_OOM) return status;
    VX_POOL_TRY(launch_apply_correction(s), "pool correction");
    VX_POOL_TRY(cudaStreamSynchronize(s->stream), "pool pass");
    if (out)
        for (uint32_t k = 0; k < p->slots; ++k)
            if (on[k]) out[k].kernel_launches = s->launches + 1;
    if (status == VX_NOT_CONVERGED) set_error("vx_pool_pass: a scene did not converge within its iteration cap");
    else if (status == VX_NONFINITE) set_error("vx_pool_pass: non-finite value in a scene's solve");
    return status;
}

int32_t vx_pool_bond_stress(vx_pool* p, uint32_t slot, float* ratio, float* force, uint32_t* near, uint32_t cap,
                            uint32_t* near_count) {
    clear_error();
    if (!p || slot >= p->slots || !p->used[slot]) {
        set_error("vx_pool_bond_stress: no scene in slot %u", slot);
        return VX_BAD_INPUT;
    }
    if (!p->s.assembled) {
        set_error("vx_pool_bond_stress: no pass has assembled the bonds yet");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    std::vector<uint8_t> only(p->slots, 0), on;
    only[slot] = 1;
    int32_t r = pool_select(p, only.data(), on);
    if (r != VX_OK) return r;
    vx_scene* s = &p->s;
    const size_t C = s->n, base = (size_t)p->first[slot] * 256, n = p->rev_n[slot];
    VX_POOL_TRY(launch_bond_stress(s, s->out_ratio, force ? s->out_force : nullptr, s->out_near, (uint32_t)(3 * C)),
                "pool bond stress");
    uint32_t count = 0;
    VX_POOL_TRY(cudaMemcpyAsync(&count, s->near_count, 4, cudaMemcpyDeviceToHost, s->stream), "stress");
    for (int a = 0; a < 3; ++a) {
        if (ratio)
            VX_POOL_TRY(cudaMemcpyAsync(ratio + a * n, s->out_ratio + a * C + base, n * 4, cudaMemcpyDeviceToHost, s->stream),
                        "stress");
        if (force)
            VX_POOL_TRY(cudaMemcpyAsync(force + 3 * a * n, s->out_force + 3 * (a * C + base), 3 * n * 4,
                                        cudaMemcpyDeviceToHost, s->stream), "stress");
    }
    VX_POOL_TRY(cudaStreamSynchronize(s->stream), "stress");
    uint32_t kept = 0;
    if (count) {
        std::vector<uint32_t> tmp(std::min<size_t>(count, 3 * C));
        VX_POOL_TRY(cudaMemcpy(tmp.data(), s->out_near, tmp.size() * 4, cudaMemcpyDeviceToHost), "near list");
        std::vector<uint32_t> local;
        for (uint32_t e : tmp) {
            size_t a = e / C, i = e - a * C;
            if (i >= base && i < base + n) local.push_back((uint32_t)(a * n + (i - base)));
        }
        std::sort(local.begin(), local.end());
        kept = (uint32_t)local.size();
        for (size_t k = 0; near && k < local.size() && k < cap; ++k) near[k] = local[k];
    }
    if (near_count) *near_count = kept;
    return VX_OK;
}


int32_t vx_pool_advance_targets(vx_pool* p, const uint8_t* enabled, const double* delta) {
    clear_error();
    if (!p || !delta) {
        set_error("vx_pool_advance_targets: null argument");
        return VX_BAD_INPUT;
    }
    for (size_t t = 0; t < 3 * (size_t)p->slots; ++t)
        if (!std::isfinite(delta[t])) {
            set_error("vx_pool_advance_targets: non-finite delta at %zu", t);
            return VX_NONFINITE;
        }
    if (p->slots > p->s.n) {  // the staging below holds 3 doubles per REV of capacity
        set_error("vx_pool_advance_targets: pool has more slots (%u) than REVs (%u)", p->slots, p->s.n);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    std::vector<uint8_t> on;
    int32_t r = pool_select(p, enabled, on);
    if (r != VX_OK) return r;
    vx_scene* s = &p->s;
    // the FP64 z vector (3 x capacity doubles, free between passes) holds the deltas
    VX_POOL_TRY(cudaStreamSynchronize(s->stream), "advance targets");
    std::memcpy(s->h_stage, delta, 3 * (size_t)p->slots * sizeof(double));
    VX_POOL_TRY(cudaMemcpyAsync(s->z64, s->h_stage, 3 * (size_t)p->slots * sizeof(double), cudaMemcpyHostToDevice,
                                s->stream), "advance targets");
    VX_POOL_TRY(launch_advance_targets(s, s->z64), "advance targets");
    VX_POOL_TRY(cudaStreamSynchronize(s->stream), "advance targets");
    return VX_OK;
}

// The fixed step of vx_scene_step for every selected slot together: each
// substep predicts the selected slots, fits, runs up to
// corotation_iterations pool passes (a slot leaves the remaining passes of
// the substep once its angle change and pass residual are within tolerance,
// src/solver.rs:561-570) and updates the velocities.
int32_t vx_pool_step(vx_pool* p, const uint8_t* enabled, const vx_step_params* prm, vx_step_stats* out) {
    clear_error();
    if (!p || !prm) {
        set_error("vx_pool_step: null argument");
        return VX_BAD_INPUT;
    }
    if (!(prm->fixed_dt > 0.0) || !std::isfinite(prm->fixed_dt) || prm->substeps == 0 ||
        prm->corotation_iterations == 0 || !std::isfinite(prm->gravity[0]) || !std::isfinite(prm->gravity[1]) ||
        !std::isfinite(prm->gravity[2])) {
        set_error("vx_pool_step: invalid fixed_dt=%g, substeps=%u, corotation_iterations=%u or gravity",
                  prm->fixed_dt, prm->substeps, prm->corotation_iterations);
        return VX_BAD_INPUT;
    }
    if (prm->contact && (!(prm->restitution >= 0.0 && prm->restitution <= 1.0) || !(prm->friction >= 0.0) ||
                         !std::isfinite(prm->friction))) {
        set_error("vx_pool_step: invalid restitution=%g or friction=%g", prm->restitution, prm->friction);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(p->s.device);
    const uint32_t S = p->slots;
    const double h = prm->fixed_dt / (double)prm->substeps;
    std::vector<uint8_t> on(S), active(S);
    for (uint32_t k = 0; k < S; ++k) on[k] = p->used[k] && (!enabled || enabled[k]);
    std::vector<vx_step_stats> st(S);
    for (uint32_t k = 0; k < S; ++k) st[k].converged = 1;
    std::vector<vx_pass_stats> ps(S);
    std::vector<double> angle(S, 0.0);
    std::vector<uint32_t> slot_contacts(S, 0);
    int32_t worst = VX_OK;
    std::vector<uint8_t> sel;
    for (uint32_t sub = 0; sub < prm->substeps; ++sub) {
        int32_t r = pool_select(p, on.data(), sel);
        if (r != VX_OK) return r;
        VX_POOL_TRY(launch_predict(&p->s, prm->gravity, h), "pool prediction");
        r = vx_pool_fit_rotations(p, on.data(), angle.data());
        if (r != VX_OK) return r;
        for (uint32_t k = 0; k < S; ++k) {
            active[k] = on[k];
            if (on[k]) st[k].max_angle = angle[k];
        }
        for (uint32_t pass = 0; pass < prm->corotation_iterations; ++pass) {
            vx_pass_params pp = prm->pass;
            pp.h = h;
            pp.reuse_preconditioner = prm->pass.reuse_preconditioner && pass > 0;
            r = vx_pool_pass(p, active.data(), &pp, ps.data());
            if (r == VX_CUDA_ERROR || r == VX_OOM || r == VX_BAD_INPUT || r == VX_TIMEOUT) return r;
            for (uint32_t k = 0; k < S; ++k) {
                if (!active[k]) continue;
                st[k].passes += 1;
                st[k].pcg_iterations += ps[k].iterations;
                st[k].residual = ps[k].residual;
                if (!ps[k].converged) {
                    st[k].converged = 0;
                    if (worst == VX_OK) worst = VX_NOT_CONVERGED;
                }
            }
            if (pass + 1 == prm->corotation_iterations) break;
            r = vx_pool_fit_rotations(p, active.data(), angle.data());
            if (r != VX_OK) return r;
            bool any = false;
            for (uint32_t k = 0; k < S; ++k) {
                if (!active[k]) continue;
                st[k].max_angle = angle[k];
                if (angle[k] <= prm->corotation_tolerance && st[k].residual <= prm->pass.tolerance) active[k] = 0;
                any = any || active[k];
            }
            if (!any) break;
        }
        r = pool_select(p, on.data(), sel);
        if (r != VX_OK) return r;
        // the order of the single-scene step: velocities from the solved
        // positions, contact projection, fracture, contact velocities
        VX_POOL_TRY(launch_velocity(&p->s, h), "pool velocity update");
        if (prm->contact) {  // every selected slot projected on its own; counts per slot
            vx_contact_stats cs{};
            r = contact_project(&p->s, &cs, slot_contacts.data());
            if (r != VX_OK) return r;
            for (uint32_t k = 0; k < S; ++k)
                if (on[k]) st[k].contacts += slot_contacts[k];
        }
        if (prm->fracture) {  // one stage over every selected slot; totals are pool-wide
            vx_dissipation d{};
            uint32_t broken = 0;
            r = fracture_stage(&p->s, h, &prm->fracture_config, &d, &broken);
            if (r != VX_OK) return r;
            for (uint32_t k = 0; k < S; ++k)
                if (on[k]) st[k].broken += broken;
        }
        if (prm->contact) {  // heat totals are pool-wide, like the broken count
            vx_contact_heat heat{};
            r = contact_resolve(&p->s, p->s.drift, prm->restitution, prm->friction, &heat);
            if (r != VX_OK) return r;
            for (uint32_t k = 0; k < S; ++k)
                if (on[k]) {
                    st[k].restitution_heat += heat.restitution;
                    st[k].friction_heat += heat.friction;
                }
        }
        VX_POOL_TRY(cudaStreamSynchronize(p->s.stream), "pool step");
    }
    if (out)
        for (uint32_t k = 0; k < S; ++k) out[k] = on[k] ? st[k] : vx_step_stats{};
    if (worst == VX_NOT_CONVERGED) set_error("vx_pool_step: a scene's pass did not reach its tolerance");
    return worst;
}

}  // extern "C"
