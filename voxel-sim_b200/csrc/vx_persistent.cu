// vx_persistent.cu — the FP32 inner PCG solve as one persistent kernel whose
// working set stays on chip.
//
// When a scene is small enough (up to ~2,000 REVs per SM), one cooperative
// block per SM (512, 608, 768 or 896 threads: the form's block size) owns a
// contiguous range of REVs for the whole inner solve. Shared memory holds, per
// REV of the range, the stiffness of its three owned bonds, a float4 + float2
// record of the iteration's vectors, its six neighbour deltas as int16, its
// mass term m/h^2 and its free-axis flags, so an in-range neighbour costs
// vector loads from shared memory and no index load. x, r, p and Ap live in
// registers of the owning thread. The operator is the FP32 row of apply_row
// (vx_pcg_core.cuh): the diagonal comes from the mass term and the bonds, so
// only its inverse is read from L2. Neighbours outside the range are read from
// a global copy that every block republishes once per iteration. An iteration
// is the recurrence of k_matvec/k_update in vx_pcg.cu (src/solver.rs:1833-1911)
// with two grid-wide reductions.
//
// One scene: neighbours read z alone, and Ap is formed as A z + beta Ap_old
// (A is linear, its projection included). The part of A z that needs only the
// block's own z (the mass term and the in-range bonds) is computed after the
// block has arrived at reduction B and before it waits there; the out-of-range
// bonds are added once B has made every block's z visible:
//   matvec phase  p = z + beta p_old, Ap += out-of-range bonds, p.Ap -> reduction A
//   update phase  alpha, x, r, z = D^-1 r, partials of r.z, r.r     -> reduction B
//                 (arrival, the in-range part of A z, the wait)
// Pools (MULTI): neighbours read the pair (z, p_old) and form p_j themselves:
//   matvec phase  p = z + beta p_old, Ap, block partial of p.Ap   -> reduction A
//   update phase  alpha, x, r, z = D^-1 r, partials of r.z, r.r   -> reduction B
// A reduction is also the grid barrier: a block stores its partial, adds one
// to an arrival counter with release semantics and polls the counter with
// acquire loads until every block has arrived; then one warp sums the
// partials in block order, so all blocks take the same alpha, beta and stop
// decisions. The per-REV dot products are formed in FP32 and summed in FP64.
// The waits are bounded; when a bound is hit the kernel records VX_TIMEOUT
// and every block leaves its loop at its next reduction.
#include <cstdlib>
#include <cstring>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_grid.cuh"
#include "vx_layout.cuh"

namespace vx {

namespace {

constexpr int kPThreads = 512;  // the pool waves' and the default range plan's block size
// shared memory per REV: K float4[3] + float2[3], (z, p_old) float4 + float2,
// three delta words, the mass term and one flag byte
constexpr int kBytesPerRev = 3 * 16 + 3 * 8 + 16 + 8 + 12 + 4 + 1;
// REVs per block at most when a pool's slots are packed into waves
// (1,536 x 113 B = 174 KB of shared memory, three REVs per thread)
constexpr uint32_t kPoolBlockRevs = 1536;

struct PersistArgs {
    uint32_t n;
    uint32_t cap;  // REVs per block (contiguous range)
    uint32_t kn;   // REV stride of the per-axis K arrays
    const uint8_t* flags;
    const float* mh2;           // m/h^2 [n]
    const float* K;
    const float* Dinv;
    const uint32_t* code;       // [3][n] neighbour deltas
    const double* src;          // right-hand side in FP64
    const double* scale_from;   // |src|; r0 = src / |src|
    float* x;                   // correction [3][n]
    float4* zp4;                // published (z.x, z.y, z.z, p_old.x) [n]
    float2* zp2;                // published (p_old.y, p_old.z) [n]
    double* part;               // [3][G] partials: p.Ap, r.z, r.r
    unsigned long long* count;  // arrivals at the grid reductions so far
    int32_t* err;               // a wait ran out
    PcgScalars* sc;
    double tolerance;
    uint32_t max_iterations;
    unsigned long long spin_limit;
    // pools: one row per block (first REV, REV count, slot, first block of the
    // slot << 16 | blocks of the slot) and the slots' states; null for one scene
    const uint4* blocks;
    SlotState* st;
};

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 smul(const Sym<float>& s, F3 v) {
    return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
            s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
__device__ __forceinline__ Sym<float> sym_of(float4 a, float2 b) { return {a.x, a.y, a.z, a.w, b.x, b.y}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// R REVs per thread. With R <= 2 the inverse diagonal block is loaded into
// registers before the grid wait of the matvec phase, so its L2 latency
// overlaps the wait; at R = 3 and 4, and for one scene at 896 threads, the
// registers are not there and it is loaded where used.
// MULTI: the blocks work for several pool slots (a.blocks, a.st); otherwise
// for one scene, whose reductions are grid_reduce's.
// TH threads per block: the register budget is 65,536 / TH (128 at 512, 107 at
// 608, 85 at 768, 73 at 896), which holds R = 4, 3, 1 and 2 REVs per thread
// without spills.
template <int R, bool MULTI, int TH = kPThreads>
__global__ void __launch_bounds__(TH, 1) k_pcg_persistent(PersistArgs a) {
    constexpr bool kPrefetch = R <= 2 && (MULTI || TH != 896);
    extern __shared__ float4 smem4[];
    __shared__ double red[3][32];
    __shared__ double tot[4];
    __shared__ int s_ok;
    const uint32_t n = a.n, cap = a.cap, T = blockDim.x;
    float4* sK4 = smem4;                                       // [3][cap] owned bonds (xx, yy, zz, xy)
    float4* sZP4 = sK4 + 3 * cap;                              // [cap] (z, p_old.x)
    float2* sK2 = reinterpret_cast<float2*>(sZP4 + cap);       // [3][cap] (xz, yz)
    float2* sZP2 = sK2 + 3 * cap;                              // [cap] (p_old.y, p_old.z)
    uint32_t* sNB = reinterpret_cast<uint32_t*>(sZP2 + cap);   // [3][cap] neighbour deltas
    float* sM = reinterpret_cast<float*>(sNB + 3 * cap);       // [cap] m/h^2
    uint8_t* sFL = reinterpret_cast<uint8_t*>(sM + cap);       // [cap] free-axis flags
    // this block's range and problem: the whole grid for one scene, or one
    // slot's blocks in a pool (its own target, iteration cap and outcome)
    uint32_t lo, cnt, slot = 0, fb = 0, nb = gridDim.x;
    double scale_norm, tolerance;
    uint32_t max_iterations;
    bool mine = true;  // this block's problem still iterates
    if constexpr (MULTI) {
        const uint4 bi = a.blocks[blockIdx.x];
        lo = bi.x, cnt = bi.y, slot = bi.z, fb = bi.w >> 16, nb = bi.w & 0xFFFFu;
        const SlotState& S = a.st[slot];
        mine = S.enabled && S.inner_on;
        scale_norm = S.r64_norm, tolerance = S.tol_in, max_iterations = S.max_its;
        if (!mine) cnt = 0;
    } else {
        lo = blockIdx.x * cap;
        cnt = lo < n ? (n - lo < cap ? n - lo : cap) : 0;
        scale_norm = *a.scale_from, tolerance = a.tolerance, max_iterations = a.max_iterations;
    }

    for (uint32_t li = threadIdx.x; li < cnt; li += T) {
        const size_t i = lo + li;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float* kb = a.K + (size_t)ax * 6 * a.kn;
            sK4[ax * cap + li] = __ldg(reinterpret_cast<const float4*>(kb) + i);
            sK2[ax * cap + li] = __ldg(reinterpret_cast<const float2*>(kb + 4 * (size_t)a.kn) + i);
            sNB[ax * cap + li] = __ldg(a.code + (size_t)ax * n + i);
        }
        sM[li] = __ldg(a.mh2 + i);
        sFL[li] = __ldg(a.flags + i);
    }

    if constexpr (!MULTI) {
        // One scene. The direction's product is formed as q = A z + beta q_old
        // (A is linear, its projection included), so the part of A z that
        // needs only this block's z (the mass term and the in-range bonds) is
        // computed between the block's arrival at the r.z reduction and its
        // wait there; the out-of-range bonds are added after the reduction
        // has made every block's z visible. Neighbours read z alone: from
        // shared memory in range (sZP4 .xyz) and from the global copy (zp4,
        // (z, 0)) outside it. The in-range part w waits in the REV's own
        // shared slots, sZP4.w and sZP2, which neighbours do not read.
        float x[R][3], r[R][3], p[R][3], q[R][3];
        Sym<float> ireg[kPrefetch ? R : 1];
        const double scale = scale_norm > 0.0 ? 1.0 / scale_norm : 1.0;
        // w = m/h^2 z + sum over in-range bonds of K (z_i - z_j), before the projection
        auto in_range = [&]() {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li >= cnt) continue;
                const uint32_t i = lo + li;
                const float4 zi = sZP4[li];
                const float mh = sM[li];
                F3 s = {mh * zi.x, mh * zi.y, mh * zi.z};
#pragma unroll
                for (int t = 0; t < 6; ++t) {
                    const uint32_t c = sNB[(t >> 1) * cap + li];
                    const int32_t dl = (int32_t)(int16_t)((t & 1) ? (c >> 16) : (c & 0xffffu));
                    const uint32_t lj = (uint32_t)((int32_t)i + dl) - lo;
                    if (lj >= cnt) continue;
                    const int ax = t < 3 ? t : t - 3;
                    const uint32_t ks = ax * cap + (t < 3 ? li : lj);
                    const Sym<float> Kb = sym_of(sK4[ks], sK2[ks]);
                    const float4 zj = sZP4[lj];
                    // a missing neighbour has delta 0: j = i and d = 0 exactly
                    const F3 kv = smul(Kb, F3{zi.x - zj.x, zi.y - zj.y, zi.z - zj.z});
                    s.x += kv.x, s.y += kv.y, s.z += kv.z;
                }
                reinterpret_cast<float*>(sZP4 + li)[3] = s.x;
                sZP2[li] = make_float2(s.y, s.z);
            }
        };
        double acc[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
#pragma unroll
            for (int c = 0; c < 3; ++c) x[k][c] = p[k][c] = q[k][c] = r[k][c] = 0.f;
            if (li < cnt) {
                const size_t i = lo + li;
                const F3 rr = {(float)(a.src[i] * scale), (float)(a.src[n + i] * scale),
                               (float)(a.src[2 * (size_t)n + i] * scale)};
                const F3 z = smul(load_sym(a.Dinv, n, i), rr);
                r[k][0] = rr.x, r[k][1] = rr.y, r[k][2] = rr.z;
                const float4 z4 = make_float4(z.x, z.y, z.z, 0.f);
                sZP4[li] = z4;
                a.zp4[i] = z4;
                acc[0] += (double)dot3(rr, z);
                acc[1] += (double)dot3(rr, rr);
            }
        }
        unsigned long long seq = 1;
        const int su[2] = {1, 2};
        const int sm[1] = {0};
        double t2[2];
        grid_arrive<2>(acc, su, a, red);
        in_range();
        const bool alive = grid_complete<2>(su, a, seq++, tot, &s_ok, t2);
        const double initial = sqrt(t2[1]);
        double rz = t2[0], rz_prev = INFINITY, residual = 0.0;
        uint32_t its = 0;
        int32_t status = alive ? VX_OK : VX_TIMEOUT;
        if (alive) {
            if (!isfinite(t2[0]) || !isfinite(t2[1])) {
                mine = false;
                status = VX_NONFINITE;
            } else if (!(initial > 1e-12)) {
                mine = false;
            } else if (max_iterations == 0) {
                mine = false;
                status = VX_NOT_CONVERGED;
            }
        }
        while (alive && mine) {
            const float beta = its == 0 ? 0.f : (float)(rz / rz_prev);
            // ---- matvec phase: p = z + beta p_old, q = A z + beta q_old ----
            double pq[1] = {0.0};
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li >= cnt) continue;
                const uint32_t i = lo + li;
                const float4 zi = sZP4[li];  // (z, w.x)
                const float2 wyz = sZP2[li];
                F3 s = {zi.w, wyz.x, wyz.y};
#pragma unroll
                for (int t = 0; t < 6; ++t) {
                    const uint32_t c = sNB[(t >> 1) * cap + li];
                    const int32_t dl = (int32_t)(int16_t)((t & 1) ? (c >> 16) : (c & 0xffffu));
                    const uint32_t j = (uint32_t)((int32_t)i + dl);
                    if (j - lo < cnt) continue;
                    const int ax = t < 3 ? t : t - 3;
                    const Sym<float> Kb = t < 3 ? sym_of(sK4[ax * cap + li], sK2[ax * cap + li])
                                                : load_sym(a.K + (size_t)ax * 6 * a.kn, a.kn, j);
                    const float4 zj = __ldcg(a.zp4 + j);
                    const F3 kv = smul(Kb, F3{zi.x - zj.x, zi.y - zj.y, zi.z - zj.z});
                    s.x += kv.x, s.y += kv.y, s.z += kv.z;
                }
                const uint8_t fl = sFL[li];
                const F3 y = {(fl & 1) ? s.x : zi.x, (fl & 2) ? s.y : zi.y, (fl & 4) ? s.z : zi.z};
                p[k][0] = fmaf(beta, p[k][0], zi.x), p[k][1] = fmaf(beta, p[k][1], zi.y),
                p[k][2] = fmaf(beta, p[k][2], zi.z);
                q[k][0] = fmaf(beta, q[k][0], y.x), q[k][1] = fmaf(beta, q[k][1], y.y),
                q[k][2] = fmaf(beta, q[k][2], y.z);
                pq[0] += (double)dot3(F3{p[k][0], p[k][1], p[k][2]}, F3{q[k][0], q[k][1], q[k][2]});
            }
            if constexpr (kPrefetch) {
#pragma unroll
                for (int k = 0; k < R; ++k) {  // in flight during the wait below
                    const uint32_t li = threadIdx.x + k * T;
                    if (li < cnt) ireg[k] = load_sym(a.Dinv, n, lo + li);
                }
            }
            double t1[1];
            if (!grid_reduce<1>(pq, sm, a, seq++, red, tot, &s_ok, t1)) {
                status = VX_TIMEOUT;
                break;
            }
            const double pq_all = t1[0];
            if (!isfinite(pq_all) || pq_all <= 1e-30) {
                its += 1;  // the matvec happened (src/solver.rs:1861-1866)
                if (!isfinite(pq_all)) status = VX_NONFINITE;
                break;
            }
            const float alpha = (float)(rz / pq_all);
            // ---- update phase; every block has read the old z: publish the new ----
            double au[2] = {0.0, 0.0};
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li >= cnt) continue;
                const size_t i = lo + li;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    x[k][c] = fmaf(alpha, p[k][c], x[k][c]);
                    r[k][c] = fmaf(-alpha, q[k][c], r[k][c]);
                }
                const F3 rr = {r[k][0], r[k][1], r[k][2]};
                Sym<float> Di;
                if constexpr (kPrefetch) Di = ireg[k];
                else Di = load_sym(a.Dinv, n, i);
                const F3 z = smul(Di, rr);
                const float4 z4 = make_float4(z.x, z.y, z.z, 0.f);
                sZP4[li] = z4;
                a.zp4[i] = z4;
                au[0] += (double)dot3(rr, z);
                au[1] += (double)dot3(rr, rr);
            }
            double tu[2];
            grid_arrive<2>(au, su, a, red);
            in_range();  // overlaps the other blocks' arrivals
            if (!grid_complete<2>(su, a, seq++, tot, &s_ok, tu)) {
                status = VX_TIMEOUT;
                break;
            }
            its += 1;
            residual = sqrt(tu[1]) / initial;
            if (!isfinite(tu[0]) || !isfinite(tu[1])) {
                status = VX_NONFINITE;
                mine = false;
            } else if (residual < tolerance) {
                mine = false;
            } else if (its >= max_iterations) {
                status = VX_NOT_CONVERGED;
                mine = false;
            }
            rz_prev = rz;
            rz = tu[0];
        }
        if (*(volatile int32_t*)a.err) status = VX_TIMEOUT;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt) continue;
            const size_t i = lo + li;
            a.x[i] = x[k][0], a.x[n + i] = x[k][1], a.x[2 * (size_t)n + i] = x[k][2];
        }
        if (threadIdx.x == 0 && blockIdx.x == 0) {
            PcgScalars* sc = a.sc;
            sc->iterations = its;
            sc->residual = residual;
            sc->initial = initial;
            sc->status = status;
            sc->done = 1;
        }
    } else {
        float x[R][3], r[R][3], p[R][3], ap[R][3];
        Sym<float> ireg[kPrefetch ? R : 1];
        const double scale = scale_norm > 0.0 ? 1.0 / scale_norm : 1.0;
        double acc[2] = {0.0, 0.0};
    #pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
    #pragma unroll
            for (int c = 0; c < 3; ++c) x[k][c] = p[k][c] = ap[k][c] = r[k][c] = 0.f;
            if (li < cnt) {
                const size_t i = lo + li;
                const F3 rr = {(float)(a.src[i] * scale), (float)(a.src[n + i] * scale),
                               (float)(a.src[2 * (size_t)n + i] * scale)};
                const F3 z = smul(load_sym(a.Dinv, n, i), rr);
                r[k][0] = rr.x, r[k][1] = rr.y, r[k][2] = rr.z;
                const float4 q4 = make_float4(z.x, z.y, z.z, 0.f);
                const float2 q2 = make_float2(0.f, 0.f);
                sZP4[li] = q4, sZP2[li] = q2;
                a.zp4[i] = q4, a.zp2[i] = q2;
                acc[0] += (double)dot3(rr, z);
                acc[1] += (double)dot3(rr, rr);
            }
        }
        unsigned long long seq = 1;
        const int su[2] = {1, 2};
        const int sm[1] = {0};
        constexpr int kActRow = 3;
        double t2[2], act = 0.0;
        // only the matvec-phase reductions carry the count of working blocks (row
        // kActRow): two of them always have a reduction, so a grid barrier, between
        bool alive;
        if constexpr (MULTI) alive = grid_reduce_ranged<2>(acc, 0.0, su, -1, a, seq++, fb, nb, red, tot, &s_ok, t2, &act);
        else alive = grid_reduce<2>(acc, su, a, seq++, red, tot, &s_ok, t2);
        const double initial = sqrt(t2[1]);
        double rz = t2[0], rz_prev = INFINITY, residual = 0.0;
        uint32_t its = 0;
        int32_t status = alive ? VX_OK : VX_TIMEOUT;
        if (alive && mine) {
            if (!isfinite(t2[0]) || !isfinite(t2[1])) {
                mine = false;
                status = VX_NONFINITE;
            } else if (!(initial > 1e-12)) {
                mine = false;
            } else if (max_iterations == 0) {
                mine = false;
                status = VX_NOT_CONVERGED;
            }
        }

        // A problem that has stopped leaves its blocks idle; in a pool they keep
        // taking part in the reductions until no block of the grid has work left,
        // so every block leaves the loop at the same reduction. One scene is one
        // problem: its blocks leave together as soon as it stops.
        while (alive) {
            if (!MULTI && !mine) break;
            const float beta = its == 0 ? 0.f : (float)(rz / rz_prev);
            // ---- matvec phase: p = z + beta p_old,
            //      Ap = P (m/h^2 p + sum K (p - p_nbr)) + (I - P) p ----
            double pap[1] = {0.0};
            const uint32_t cnt_now = mine ? cnt : 0;
    #pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li >= cnt_now) continue;
                const uint32_t i = lo + li;
                int32_t dl[6];
    #pragma unroll
                for (int w = 0; w < 3; ++w) {
                    const uint32_t c = sNB[w * cap + li];
                    dl[2 * w] = (int32_t)(int16_t)(c & 0xffffu);
                    dl[2 * w + 1] = (int32_t)(int16_t)(c >> 16);
                }
                const uint8_t fl = sFL[li];
                const float4 o4 = sZP4[li];
                const float2 o2 = sZP2[li];
                const F3 pi = {fmaf(beta, o4.w, o4.x), fmaf(beta, o2.x, o4.y), fmaf(beta, o2.y, o4.z)};
                const float mh = sM[li];
                F3 s = {mh * pi.x, mh * pi.y, mh * pi.z};
    #pragma unroll
                for (int t = 0; t < 6; ++t) {
                    const uint32_t j = (uint32_t)((int32_t)i + dl[t]);
                    const int ax = t < 3 ? t : t - 3;
                    const uint32_t lj = j - lo;
                    const bool inb = lj < cnt;
                    float4 q4;
                    float2 q2;
                    Sym<float> Kb;
                    if (inb) {
                        q4 = sZP4[lj], q2 = sZP2[lj];
                    } else {
                        q4 = __ldcg(a.zp4 + j), q2 = __ldcg(a.zp2 + j);
                    }
                    if (t < 3) {
                        Kb = sym_of(sK4[ax * cap + li], sK2[ax * cap + li]);
                    } else if (inb) {
                        Kb = sym_of(sK4[ax * cap + lj], sK2[ax * cap + lj]);
                    } else {
                        Kb = load_sym(a.K + (size_t)ax * 6 * a.kn, a.kn, j);
                    }
                    const F3 pn = {fmaf(beta, q4.w, q4.x), fmaf(beta, q2.x, q4.y), fmaf(beta, q2.y, q4.z)};
                    // a missing neighbour has delta 0: j = i, pn = pi and d = 0 exactly
                    const F3 d = {pi.x - pn.x, pi.y - pn.y, pi.z - pn.z};
                    const F3 kv = smul(Kb, d);
                    s.x += kv.x, s.y += kv.y, s.z += kv.z;
                }
                const F3 y = {(fl & 1) ? s.x : pi.x, (fl & 2) ? s.y : pi.y, (fl & 4) ? s.z : pi.z};
                p[k][0] = pi.x, p[k][1] = pi.y, p[k][2] = pi.z;
                ap[k][0] = y.x, ap[k][1] = y.y, ap[k][2] = y.z;
                pap[0] += (double)dot3(pi, y);
            }
            if constexpr (kPrefetch) {
    #pragma unroll
                for (int k = 0; k < R; ++k) {  // in flight during the wait below
                    const uint32_t li = threadIdx.x + k * T;
                    if (li < cnt_now) ireg[k] = load_sym(a.Dinv, n, lo + li);
                }
            }
            double t1[1];
            bool ok_a;
            if constexpr (MULTI)
                ok_a = grid_reduce_ranged<1>(pap, mine ? 1.0 : 0.0, sm, kActRow, a, seq++, fb, nb, red, tot, &s_ok, t1, &act);
            else
                ok_a = grid_reduce<1>(pap, sm, a, seq++, red, tot, &s_ok, t1);
            if (!ok_a) {
                status = VX_TIMEOUT;
                break;
            }
            if (MULTI && act == 0.0) break;  // no block of the grid has work left
            const double pap_all = t1[0];
            if (mine && (!isfinite(pap_all) || pap_all <= 1e-30)) {
                its += 1;  // the matvec happened (src/solver.rs:1861-1866)
                if (!isfinite(pap_all)) status = VX_NONFINITE;
                mine = false;
                if (!MULTI) break;
            }
            const float alpha = mine ? (float)(rz / pap_all) : 0.f;
            // ---- update phase; every block has read the old (z, p_old): publish the new ----
            double au[2] = {0.0, 0.0};
            const uint32_t cnt_up = mine ? cnt : 0;
    #pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li >= cnt_up) continue;
                const size_t i = lo + li;
    #pragma unroll
                for (int c = 0; c < 3; ++c) {
                    x[k][c] = fmaf(alpha, p[k][c], x[k][c]);
                    r[k][c] = fmaf(-alpha, ap[k][c], r[k][c]);
                }
                const F3 rr = {r[k][0], r[k][1], r[k][2]};
                Sym<float> Di;
                if constexpr (kPrefetch) Di = ireg[k];
                else Di = load_sym(a.Dinv, n, i);
                const F3 z = smul(Di, rr);
                const float4 q4 = make_float4(z.x, z.y, z.z, p[k][0]);
                const float2 q2 = make_float2(p[k][1], p[k][2]);
                sZP4[li] = q4, sZP2[li] = q2;
                a.zp4[i] = q4, a.zp2[i] = q2;
                au[0] += (double)dot3(rr, z);
                au[1] += (double)dot3(rr, rr);
            }
            double tu[2], act_u = 0.0;
            bool ok_b;
            if constexpr (MULTI) ok_b = grid_reduce_ranged<2>(au, 0.0, su, -1, a, seq++, fb, nb, red, tot, &s_ok, tu, &act_u);
            else ok_b = grid_reduce<2>(au, su, a, seq++, red, tot, &s_ok, tu);
            if (!ok_b) {
                status = VX_TIMEOUT;
                break;
            }
            if (mine) {
                its += 1;
                residual = sqrt(tu[1]) / initial;
                if (!isfinite(tu[0]) || !isfinite(tu[1])) {
                    status = VX_NONFINITE;
                    mine = false;
                } else if (residual < tolerance) {
                    mine = false;
                } else if (its >= max_iterations) {
                    status = VX_NOT_CONVERGED;
                    mine = false;
                }
            }
            rz_prev = rz;
            rz = tu[0];
        }
        if (*(volatile int32_t*)a.err) status = VX_TIMEOUT;
    #pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt) continue;
            const size_t i = lo + li;
            a.x[i] = x[k][0], a.x[n + i] = x[k][1], a.x[2 * (size_t)n + i] = x[k][2];
        }
        if (threadIdx.x == 0 && blockIdx.x == fb) {
            if constexpr (MULTI) {
                SlotState& S = a.st[slot];
                if (S.enabled && S.inner_on) {
                    S.its = its;
                    S.residual_in = residual;
                    S.initial = initial;
                    S.status_in = status;
                    S.done = 1;
                }
            } else {
                PcgScalars* sc = a.sc;
                sc->iterations = its;
                sc->residual = residual;
                sc->initial = initial;
                sc->status = status;
                sc->done = 1;
            }
        }
    }
}

template <int R, bool MULTI, int TH = kPThreads>
cudaError_t launch_r(const PersistArgs& a, unsigned G, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_pcg_persistent<R, MULTI, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    PersistArgs args = a;
    void* params[] = {&args};
    return cudaLaunchCooperativeKernel((void*)k_pcg_persistent<R, MULTI, TH>, dim3(G), dim3(TH), params, smem, st);
}

// Threads per block of a range form, and the most REVs per thread it is built for.
unsigned range_threads(int form) {
    switch (form) {
        case VX_PERSIST_RANGE_608: return 608;
        case VX_PERSIST_RANGE_768: return 768;
        case VX_PERSIST_RANGE_896: return 896;
        default: return (unsigned)kPThreads;
    }
}
unsigned range_max_revs_per_thread(unsigned th) {
    return th <= 512 ? 4u : (th <= 608 ? 3u : (th <= 768 ? 1u : 2u));  // 2 at 768 spills
}

}  // namespace

static bool range_plan(vx_scene* s, int form);

// The on-chip form an untuned scene takes, by its REVs per block (cap): the
// fastest form measured at that cap on mixed blocks (one autotuner run at
// 24^3, 48^3 and 64^3: caps 256, 748 and 1,772): one reduction per iteration
// up to 512 REVs per block, the classic range form at 768 threads up to 768,
// at 896 threads up to 1,792, and at 512 threads above. A form that does not
// fit falls through to the next.
static bool untuned_plan(vx_scene* s) {
    unsigned G = (unsigned)s->sm_count;
    const unsigned min_blocks = (s->n + 255) / 256;
    if (min_blocks < G) G = min_blocks;
    if (G == 0) G = 1;
    const unsigned cap = (s->n + G - 1) / G;
    if (cap <= 512 && expanded_plan(s)) return true;
    if (cap <= 768 && range_plan(s, VX_PERSIST_RANGE_768)) return true;
    if (cap <= 1792 && range_plan(s, VX_PERSIST_RANGE_896)) return true;
    return range_plan(s, VX_PERSIST_RANGE) || expanded_plan(s);
}

// Whether the persistent inner solve fits this scene on this GPU; caches the
// shape. Without a chosen form the scene takes untuned_plan's form, and the
// brick plan (vx_brick.cu) where no range form fits (neighbour deltas beyond
// an int16). A chosen form (the autotuner's, or
// VXCOROT_PERSISTENT=expanded|range|range608|range768|range896|brick) is that
// form or nothing.
bool persistent_plan(vx_scene* s) {
    if (s->persist_checked) return s->persist_ok;
    s->persist_checked = true;
    s->persist_ok = false;
    s->brick_ok = false;
    s->exp_ok = false;
    if (s->n == 0) return false;
    int form = s->persist_form;
    if (const char* v = std::getenv("VXCOROT_PERSISTENT")) {
        if (std::strcmp(v, "expanded") == 0) form = VX_PERSIST_EXPANDED;
        else if (std::strcmp(v, "range") == 0) form = VX_PERSIST_RANGE;
        else if (std::strcmp(v, "range608") == 0) form = VX_PERSIST_RANGE_608;
        else if (std::strcmp(v, "range768") == 0) form = VX_PERSIST_RANGE_768;
        else if (std::strcmp(v, "range896") == 0) form = VX_PERSIST_RANGE_896;
        else if (std::strcmp(v, "brick") == 0) form = VX_PERSIST_BRICK_T1_256;
    }
    bool ok;
    if (form == VX_PERSIST_EXPANDED) ok = expanded_plan(s);
    else if (form == VX_PERSIST_RANGE || form >= VX_PERSIST_RANGE_608) ok = range_plan(s, form);
    else if (form != 0) ok = brick_plan(s, form);
    else ok = untuned_plan(s) || brick_plan(s, VX_PERSIST_BRICK_T1_256);
    s->persist_ok = ok;
    return ok;
}

// Whether every neighbour delta j - i of the scene fits an int16 (read back
// once per topology from k_neighbor_codes' flag).
bool neighbor_deltas_fit(vx_scene* s) {
    if (s->nbcode_state == 0) {
        uint32_t bad = 0;
        if (cudaMemcpyAsync(&bad, s->nbcode_bad, sizeof bad, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            return false;
        s->nbcode_state = bad == 0 ? 1 : 2;
    }
    return s->nbcode_state == 1;
}

// The contiguous-range plan: block b owns REVs [b cap, (b + 1) cap), with the
// block size of the form (range_threads).
static bool range_plan(vx_scene* s, int form) {
    if (!neighbor_deltas_fit(s)) return false;
    int dev = s->device, max_smem = 0, coop = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return false;
    unsigned G = (unsigned)s->sm_count;
    unsigned min_blocks = (s->n + 255) / 256;  // at least 256 REVs per block
    if (min_blocks < G) G = min_blocks;
    if (G == 0) G = 1;
    const unsigned TH = range_threads(form);
    unsigned cap = (s->n + G - 1) / G;
    unsigned R = (cap + TH - 1) / TH;
    size_t smem = ((size_t)kBytesPerRev * cap + 15) & ~size_t(15);
    if (R > range_max_revs_per_thread(TH) || smem + 4096 > (size_t)max_smem) return false;
    s->persist_G = G;
    s->persist_cap = cap;
    s->persist_T = TH;
    // R = 3 only at 608 threads, whose budget is built for it
    s->persist_R = R <= 1 ? 1 : (R <= 2 ? 2 : (TH == 608 ? 3 : 4));
    s->persist_smem = smem;
    return true;
}

uint32_t persistent_block_cap() { return kPoolBlockRevs; }


// One cooperative launch of the persistent inner solve over the pool slots of
// a wave: d_blocks holds one row per block (first REV, REV count, slot, first
// block of the slot << 16 | the slot's blocks); each slot solves
// A32 d = r64 / |r64| on its own REVs to its own inner target (SlotState) and
// writes its outcome there. Blocks of slots that are not iterating are idle.
int32_t solve_inner_slots(vx_scene* s, const uint4* d_blocks, SlotState* st, unsigned G, uint32_t cap) {
    int dev = s->device, max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t smem = ((size_t)kBytesPerRev * cap + 15) & ~size_t(15);
    if (cap == 0 || cap > 4u * kPThreads || G > (unsigned)s->sm_count || smem + 4096 > (size_t)max_smem) {
        set_error("persistent pool PCG: a wave of %u blocks of %u REVs does not fit", G, cap);
        return VX_BAD_INPUT;
    }
    PersistArgs a;
    a.n = s->n;
    a.cap = cap;
    a.kn = kstride32(s->n);
    a.flags = s->flags;
    a.mh2 = s->mh2_32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.code = s->nbcode;
    a.src = s->r64;
    a.scale_from = nullptr;
    a.x = s->x32;
    a.zp4 = reinterpret_cast<float4*>(s->zp32);
    a.zp2 = reinterpret_cast<float2*>(s->zp32 + 4 * (size_t)s->n);
    a.part = s->partials;
    a.count = reinterpret_cast<unsigned long long*>(s->barrier);
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = nullptr;
    a.tolerance = 0.0;
    a.max_iterations = 0;
    a.blocks = d_blocks;
    a.st = st;
    a.spin_limit = 4000000ull;
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    // one instantiation for every wave: the compiler schedules and contracts the
    // arithmetic of k_pcg_persistent<1>, <2> and <4> differently, and a slot's
    // bits must not depend on the largest block of the wave it lands in
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) e = launch_r<4, true>(a, G, smem, s->stream);
    s->launches += 1;
    if (e != cudaSuccess) {
        set_error("persistent pool PCG launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

// One FP32 inner solve A32 d = r64 / |r64| in a single cooperative launch.
int32_t solve_inner_persistent(vx_scene* s, double tolerance, uint32_t max_iterations) {
    if (s->exp_ok) return solve_inner_expanded(s, tolerance, max_iterations);
    if (s->brick_ok) return solve_inner_brick(s, tolerance, max_iterations);
    PersistArgs a;
    a.n = s->n;
    a.cap = s->persist_cap;
    a.kn = kstride32(s->n);
    a.flags = s->flags;
    a.mh2 = s->mh2_32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.code = s->nbcode;
    a.src = s->r64;
    a.scale_from = &s->sc->r64_norm;
    a.x = s->x32;
    a.zp4 = reinterpret_cast<float4*>(s->zp32);
    a.zp2 = reinterpret_cast<float2*>(s->zp32 + 4 * (size_t)s->n);
    a.part = s->partials;
    a.count = reinterpret_cast<unsigned long long*>(s->barrier);
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = s->sc32;
    a.tolerance = tolerance;
    a.max_iterations = max_iterations;
    a.blocks = nullptr;
    a.st = nullptr;
    a.spin_limit = 4000000ull;  // ~1-2 s of polling at one reduction
    // VXCOROT_BARRIER_SPINS lowers the bound so a test can make the wait run out
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) {
        const unsigned G = s->persist_G;
        const size_t sm = s->persist_smem;
        switch (s->persist_T * 8 + s->persist_R) {
            case 512 * 8 + 1: e = launch_r<1, false>(a, G, sm, s->stream); break;
            case 512 * 8 + 2: e = launch_r<2, false>(a, G, sm, s->stream); break;
            case 608 * 8 + 1: e = launch_r<1, false, 608>(a, G, sm, s->stream); break;
            case 608 * 8 + 2: e = launch_r<2, false, 608>(a, G, sm, s->stream); break;
            case 608 * 8 + 3: e = launch_r<3, false, 608>(a, G, sm, s->stream); break;
            case 768 * 8 + 1: e = launch_r<1, false, 768>(a, G, sm, s->stream); break;
            case 896 * 8 + 1: e = launch_r<1, false, 896>(a, G, sm, s->stream); break;
            case 896 * 8 + 2: e = launch_r<2, false, 896>(a, G, sm, s->stream); break;
            default: e = launch_r<4, false>(a, G, sm, s->stream); break;
        }
    }
    s->launches += 1;
    if (e != cudaSuccess) {
        set_error("persistent PCG launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

}  // namespace vx
