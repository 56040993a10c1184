// vx_pcg_core.cuh — the operator row and vector helpers shared by the
// single-scene PCG kernels (vx_pcg.cu) and the pool kernels (vx_pool.cu).
#pragma once

#include "vx_device.cuh"
#include "vx_internal.h"
#include "vx_layout.cuh"
#include "vx_reduce.cuh"

namespace vx {

template <typename T>
struct IterArgs {
    uint32_t n;
    uint32_t kn;      // REV stride of the per-axis K arrays (n in FP64, kstride32(n) in FP32)
    const uint8_t* flags;
    const T* D;       // projected diagonal (sym layout)
    const T* K;       // per-axis bond K (3 sym layouts), zero when not assembled
    const T* Dinv;
    const uint32_t* nbr;
    const uint32_t* rev;
    const float* mh2;  // FP32 form: [n] m/h^2, from which the operator forms D v
    const T* z_in;    // matvec: z
    const T* p_old;   // matvec: previous direction
    T* p_new;         // matvec: new direction
    T* ap;
    T* x;
    T* r;
    T* z;
    double* pm;       // [G] partials of p.Ap
    double* pu;       // [2][G] partials of r.z, r.r
    PcgScalars* sc;
};

template <typename T>
struct V3 {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ V3<T> mul(const Sym<T>& s, V3<T> v) {
    return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
            s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
template <typename T>
__device__ __forceinline__ V3<T> load_v(const T* p, size_t n, size_t i) {
    return {p[i], p[n + i], p[2 * n + i]};
}
template <typename T>
__device__ __forceinline__ V3<T> ldg_v(const T* __restrict__ p, size_t n, size_t i) {
    return {__ldg(p + i), __ldg(p + n + i), __ldg(p + 2 * n + i)};
}
template <typename T>
__device__ __forceinline__ void store_v(T* p, size_t n, size_t i, V3<T> v) {
    p[i] = v.x;
    p[n + i] = v.y;
    p[2 * n + i] = v.z;
}
template <typename T>
__device__ __forceinline__ double dot_d(V3<T> a, V3<T> b) {
    return (double)a.x * (double)b.x + (double)a.y * (double)b.y + (double)a.z * (double)b.z;
}

// ---- block totals of the previous kernel's partials -----------------------------
// Every thread gets the totals; the summation order is fixed (thread t adds
// partials t, t+256, ... then the block tree), identical in every block.
template <int NV>
__device__ __forceinline__ void block_total(const double* part, unsigned G, double (&out)[NV]) {
    __shared__ double sh[NV][kThreads / 32];
    __shared__ double tot[NV];
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        v[k] = 0.0;
        for (unsigned b = threadIdx.x; b < G; b += kThreads) v[k] += __ldcg(part + (size_t)k * G + b);
    }
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = tot[k];
}

template <int NV>
__device__ __forceinline__ void block_partial(double (&v)[NV], double* part, unsigned G) {
    __shared__ double sh[NV][kThreads / 32];
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) part[(size_t)k * G + blockIdx.x] = v[k];
    }
}

// ---- one row of the operator ----------------------------------------------------------
// A v at REV i, with D_i = P_i (m_i/h^2 I + sum_e K_e) P_i + (I - P_i) and the sums
// over its six bonds e (the three it owns, K_(a,i) to nbr(a), and the three owned
// by its -axis neighbours k, K_(a,k)):
//   FP64:  D_i v_i - P_i sum_e K_e v_j            (the reference's row, assembled D)
//   FP32:  P_i (m_i/h^2 v_i + sum_e K_e (v_i - v_j)) + (I - P_i) v_i
// Both are the same operator on directions that vanish on fixed axes, which the
// PCG's are (r and so z = D^-1 r are zero there). The FP32 form reads 4 bytes of
// mass term instead of the 24-byte D and never subtracts two large products, so
// a stiff lattice loses less to cancellation: on the 160^3 damaged lattice the
// refined solve needs 9 % fewer inner iterations. `get(j)` returns v_j. All
// loads are issued before the arithmetic: missing neighbours read REV i itself
// and are masked to zero.
template <typename T, typename Get>
__device__ __forceinline__ V3<T> apply_row(const IterArgs<T>& a, uint32_t i, V3<T> vi, Get get) {
    const size_t n = a.n;
    uint32_t nb[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        nb[ax] = __ldg(a.nbr + ax * n + i);
        nb[3 + ax] = __ldg(a.rev + ax * n + i);
    }
    const uint8_t fl = __ldg(a.flags + i);
    Sym<T> D;
    T mh = T(0);
    if constexpr (sizeof(T) == 4) mh = __ldg(a.mh2 + i);
    else D = load_sym(a.D, n, i);
    Sym<T> Ko[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) Ko[ax] = load_sym(a.K + (size_t)ax * 6 * a.kn, a.kn, i);
    uint32_t jj[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) jj[s] = nb[s] == VX_EMPTY_U32 ? i : nb[s];
    V3<T> vj[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) vj[s] = get(jj[s]);
    Sym<T> Kr[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) Kr[ax] = load_sym(a.K + (size_t)ax * 6 * a.kn, a.kn, jj[3 + ax]);
    if constexpr (sizeof(T) == 4) {
        V3<T> s = {mh * vi.x, mh * vi.y, mh * vi.z};
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            const bool ok = nb[t] != VX_EMPTY_U32;
            V3<T> d = ok ? V3<T>{vi.x - vj[t].x, vi.y - vj[t].y, vi.z - vj[t].z} : V3<T>{T(0), T(0), T(0)};
            V3<T> kv = mul(t < 3 ? Ko[t] : Kr[t - 3], d);
            s.x += kv.x;
            s.y += kv.y;
            s.z += kv.z;
        }
        return V3<T>{(fl & 1) ? s.x : vi.x, (fl & 2) ? s.y : vi.y, (fl & 4) ? s.z : vi.z};
    } else {
        V3<T> y = mul(D, vi);
        V3<T> s = {T(0), T(0), T(0)};
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            const bool ok = nb[t] != VX_EMPTY_U32;
            V3<T> v = ok ? vj[t] : V3<T>{T(0), T(0), T(0)};
            V3<T> kv = mul(t < 3 ? Ko[t] : Kr[t - 3], v);
            s.x += kv.x;
            s.y += kv.y;
            s.z += kv.z;
        }
        if (fl & 1) y.x -= s.x;
        if (fl & 2) y.y -= s.y;
        if (fl & 4) y.z -= s.z;
        return y;
    }
}

}  // namespace vx
