// vx_persistent.cu — the FP32 inner PCG solve as one persistent kernel whose
// working set stays on chip.
//
// When a scene is small enough (up to ~1,900 REVs per SM), one cooperative
// block of 512 threads per SM owns a contiguous range of REVs for the whole
// inner solve. Its REVs' bond stiffness (three owned bonds), projected
// diagonal, z and p live in shared memory; x, r, p and Ap live in registers
// of the owning thread. Neighbours inside the range are read from shared
// memory, the others from the global copies of z and p (L2). An iteration is
// the same recurrence as k_matvec/k_update in vx_pcg.cu (src/solver.rs:1833-1911)
// with two grid barriers:
//   matvec phase  p = z + beta p_old, Ap, block partial of p.Ap   -> barrier A
//   update phase  alpha, x, r, z = D^-1 r, partials of r.z, r.r   -> barrier B
// Every block sums the partials in the same fixed order, so all blocks take
// the same alpha, beta and stop decisions. The barriers spin a bounded number
// of times; when the bound is hit the kernel records VX_TIMEOUT and every
// block leaves its loop at its next barrier.
#include <cstdlib>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_layout.cuh"

namespace vx {

namespace {

constexpr int kPThreads = 512;
constexpr int kFloatsPerRev = 30;  // 18 K + 6 D + 3 z + 3 p in shared memory

struct PersistArgs {
    uint32_t n;
    uint32_t cap;  // REVs per block (contiguous range)
    const uint8_t* flags;
    const float* D;
    const float* K;
    const float* Dinv;
    const uint32_t* nbr;
    const uint32_t* rev;
    const double* src;         // right-hand side in FP64
    const double* scale_from;  // |src|; r0 = src / |src|
    float* x;                  // correction [3][n]
    float* zg;                 // global z [3][n]
    float* pg;                 // global p [3][n]
    double* part;              // [3][G] partials: p.Ap, r.z, r.r
    unsigned* bar;             // [2] arrival count, generation
    int32_t* err;              // barrier timeout flag
    PcgScalars* sc;
    double tolerance;
    uint32_t max_iterations;
    unsigned long long spin_limit;
};

template <int NV>
__device__ __forceinline__ void reduce_block(double (&v)[NV], double (*sh)[32]) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = warp_sum(lane < nw ? sh[k][lane] : 0.0);
    }
    __syncthreads();
}

// Sum of G partials in a fixed order; the result reaches every thread.
template <int NV>
__device__ __forceinline__ void grid_totals(const double* part, unsigned G, const int (&slot)[NV],
                                            double (*sh)[32], double* tot, double (&out)[NV]) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        v[k] = 0.0;
        for (unsigned b = threadIdx.x; b < G; b += blockDim.x) v[k] += __ldcg(part + (size_t)slot[k] * G + b);
    }
    reduce_block<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = tot[k];
}

// Generation barrier over all blocks of a cooperative launch with a bounded
// wait. Returns false (in every thread of the block) once any block has timed
// out, so the caller leaves its loop.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int32_t* err, unsigned long long spin_limit) {
    __shared__ int32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u) + 1u;
        int32_t ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long spins = 0;
            while (*gen == g0) {
                if (++spins > spin_limit) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
        if (*(volatile int32_t*)err) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 smul(const Sym<float>& s, F3 v) {
    return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
            s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
// Inverse of a symmetric positive block by its adjugate, scaled by the largest
// diagonal entry so the FP32 cofactors stay far from overflow.
__device__ __forceinline__ Sym<float> sym_inverse(const Sym<float>& d) {
    const float s = fmaxf(fmaxf(d.xx, d.yy), d.zz);
    const float is = 1.0f / s;
    const float xx = d.xx * is, yy = d.yy * is, zz = d.zz * is, xy = d.xy * is, xz = d.xz * is, yz = d.yz * is;
    const float c00 = yy * zz - yz * yz, c01 = xz * yz - xy * zz, c02 = xy * yz - xz * yy;
    const float c11 = xx * zz - xz * xz, c12 = xy * xz - xx * yz, c22 = xx * yy - xy * xy;
    const float inv = is / (xx * c00 + xy * c01 + xz * c02);
    return {c00 * inv, c11 * inv, c22 * inv, c01 * inv, c02 * inv, c12 * inv};
}
__device__ __forceinline__ Sym<float> ssym(const float* base, uint32_t cap, uint32_t li) {
    return {base[li], base[cap + li], base[2 * cap + li], base[3 * cap + li], base[4 * cap + li], base[5 * cap + li]};
}
__device__ __forceinline__ F3 s3(const float* base, uint32_t cap, uint32_t li) {
    return {base[li], base[cap + li], base[2 * cap + li]};
}
__device__ __forceinline__ void w3(float* base, uint32_t cap, uint32_t li, F3 v) {
    base[li] = v.x;
    base[cap + li] = v.y;
    base[2 * cap + li] = v.z;
}

template <int R>
__global__ void __launch_bounds__(kPThreads, 1) k_pcg_persistent(PersistArgs a) {
    extern __shared__ float smem[];
    __shared__ double red[3][32];
    __shared__ double tot[3];
    const uint32_t n = a.n, cap = a.cap, T = blockDim.x, G = gridDim.x;
    float* sK = smem;             // [18][cap]: axis a component c at (6a + c) * cap
    float* sD = sK + 18 * cap;    // [6][cap]
    float* sz = sD + 6 * cap;     // [3][cap]
    float* sp = sz + 3 * cap;     // [3][cap]
    const uint32_t lo = blockIdx.x * cap;
    const uint32_t cnt = lo < n ? (n - lo < cap ? n - lo : cap) : 0;

    // stiffness and diagonal of the range into shared memory
    for (uint32_t li = threadIdx.x; li < cnt; li += T) {
        const uint32_t i = lo + li;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            Sym<float> k = load_sym(a.K + (size_t)ax * 6 * n, n, i);
            float* b = sK + (size_t)6 * ax * cap;
            b[li] = k.xx, b[cap + li] = k.yy, b[2 * cap + li] = k.zz;
            b[3 * cap + li] = k.xy, b[4 * cap + li] = k.xz, b[5 * cap + li] = k.yz;
        }
        Sym<float> d = load_sym(a.D, n, i);
        sD[li] = d.xx, sD[cap + li] = d.yy, sD[2 * cap + li] = d.zz;
        sD[3 * cap + li] = d.xy, sD[4 * cap + li] = d.xz, sD[5 * cap + li] = d.yz;
    }

    float x[R][3], r[R][3], p[R][3], ap[R][3];
    double scale = 1.0;
    {
        double rn = *a.scale_from;
        scale = rn > 0.0 ? 1.0 / rn : 1.0;
    }
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t li = threadIdx.x + k * T;
        x[k][0] = x[k][1] = x[k][2] = 0.f;
        p[k][0] = p[k][1] = p[k][2] = 0.f;
        ap[k][0] = ap[k][1] = ap[k][2] = 0.f;
        r[k][0] = r[k][1] = r[k][2] = 0.f;
        if (li < cnt) {
            const size_t i = lo + li;
            F3 rr = {(float)(a.src[i] * scale), (float)(a.src[n + i] * scale), (float)(a.src[2 * (size_t)n + i] * scale)};
            F3 z = smul(load_sym(a.Dinv, n, i), rr);
            r[k][0] = rr.x, r[k][1] = rr.y, r[k][2] = rr.z;
            w3(sz, cap, li, z);
            w3(sp, cap, li, F3{0.f, 0.f, 0.f});
            a.zg[i] = z.x, a.zg[n + i] = z.y, a.zg[2 * (size_t)n + i] = z.z;
            a.pg[i] = 0.f, a.pg[n + i] = 0.f, a.pg[2 * (size_t)n + i] = 0.f;
            acc[0] += (double)rr.x * z.x + (double)rr.y * z.y + (double)rr.z * z.z;
            acc[1] += (double)rr.x * rr.x + (double)rr.y * rr.y + (double)rr.z * rr.z;
        }
    }
    reduce_block<2>(acc, red);
    if (threadIdx.x == 0) {
        a.part[(size_t)1 * G + blockIdx.x] = acc[0];
        a.part[(size_t)2 * G + blockIdx.x] = acc[1];
    }
    bool alive = grid_barrier(a.bar, a.err, a.spin_limit);
    double t2[2] = {0.0, 0.0};
    const int su[2] = {1, 2};
    if (alive) grid_totals<2>(a.part, G, su, red, tot, t2);
    const double initial = sqrt(t2[1]);
    double rz = t2[0], rz_prev = INFINITY, residual = 0.0;
    uint32_t its = 0;
    int32_t status = VX_OK;
    bool done = !alive;
    if (alive) {
        if (!isfinite(t2[0]) || !isfinite(t2[1])) {
            done = true;
            status = VX_NONFINITE;
        } else if (!(initial > 1e-12)) {
            done = true;
        } else if (a.max_iterations == 0) {
            done = true;
            status = VX_NOT_CONVERGED;
        }
    }

    while (!done) {
        const float beta = its == 0 ? 0.f : (float)(rz / rz_prev);
        // ---- matvec phase: p = z + beta p_old, Ap = D p - P sum K p_nbr ----
        double pap = 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt) continue;
            const uint32_t i = lo + li;
            uint32_t nb[6];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                nb[ax] = __ldg(a.nbr + (size_t)ax * n + i);
                nb[3 + ax] = __ldg(a.rev + (size_t)ax * n + i);
            }
            const uint8_t fl = __ldg(a.flags + i);
            F3 zi = s3(sz, cap, li), po = s3(sp, cap, li);
            F3 pi = {fmaf(beta, po.x, zi.x), fmaf(beta, po.y, zi.y), fmaf(beta, po.z, zi.z)};
            F3 y = smul(ssym(sD, cap, li), pi);
            F3 s = {0.f, 0.f, 0.f};
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const uint32_t jraw = nb[t];
                const bool ok = jraw != VX_EMPTY_U32;
                const uint32_t j = ok ? jraw : i;
                const int ax = t < 3 ? t : t - 3;
                const uint32_t lj = j - lo;
                const bool inb = lj < cnt;
                const uint32_t ls = inb ? lj : li;  // always a valid shared-memory slot
                F3 zj = s3(sz, cap, ls), pj = s3(sp, cap, ls);
                Sym<float> Kb = ssym(sK + (size_t)6 * ax * cap, cap, t < 3 ? li : ls);
                if (!inb) {
                    zj = {__ldcg(a.zg + j), __ldcg(a.zg + n + j), __ldcg(a.zg + 2 * (size_t)n + j)};
                    pj = {__ldcg(a.pg + j), __ldcg(a.pg + n + j), __ldcg(a.pg + 2 * (size_t)n + j)};
                    if (t >= 3) Kb = load_sym(a.K + (size_t)ax * 6 * n, n, j);
                }
                const float m = ok ? 1.f : 0.f;
                F3 pn = {m * fmaf(beta, pj.x, zj.x), m * fmaf(beta, pj.y, zj.y), m * fmaf(beta, pj.z, zj.z)};
                F3 kv = smul(Kb, pn);
                s.x += kv.x, s.y += kv.y, s.z += kv.z;
            }
            if (fl & 1) y.x -= s.x;
            if (fl & 2) y.y -= s.y;
            if (fl & 4) y.z -= s.z;
            p[k][0] = pi.x, p[k][1] = pi.y, p[k][2] = pi.z;
            ap[k][0] = y.x, ap[k][1] = y.y, ap[k][2] = y.z;
            pap += (double)pi.x * y.x + (double)pi.y * y.y + (double)pi.z * y.z;
        }
        double v1[1] = {pap};
        reduce_block<1>(v1, red);
        if (threadIdx.x == 0) a.part[blockIdx.x] = v1[0];
        if (!grid_barrier(a.bar, a.err, a.spin_limit)) {
            status = VX_TIMEOUT;
            break;
        }
        // every block has read the old directions: publish the new ones
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt) continue;
            const size_t i = lo + li;
            w3(sp, cap, li, F3{p[k][0], p[k][1], p[k][2]});
            a.pg[i] = p[k][0], a.pg[n + i] = p[k][1], a.pg[2 * (size_t)n + i] = p[k][2];
        }
        double t1[1];
        const int sm[1] = {0};
        grid_totals<1>(a.part, G, sm, red, tot, t1);
        const double pap_all = t1[0];
        if (!isfinite(pap_all) || pap_all <= 1e-30) {
            its += 1;  // the matvec happened (src/solver.rs:1861-1866)
            if (!isfinite(pap_all)) status = VX_NONFINITE;
            break;
        }
        const float alpha = (float)(rz / pap_all);
        // ---- update phase ----
        double au[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt) continue;
            const size_t i = lo + li;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                x[k][c] = fmaf(alpha, p[k][c], x[k][c]);
                r[k][c] = fmaf(-alpha, ap[k][c], r[k][c]);
            }
            F3 rr = {r[k][0], r[k][1], r[k][2]};
            F3 z = smul(sym_inverse(ssym(sD, cap, li)), rr);
            w3(sz, cap, li, z);
            a.zg[i] = z.x, a.zg[n + i] = z.y, a.zg[2 * (size_t)n + i] = z.z;
            au[0] += (double)rr.x * z.x + (double)rr.y * z.y + (double)rr.z * z.z;
            au[1] += (double)rr.x * rr.x + (double)rr.y * rr.y + (double)rr.z * rr.z;
        }
        reduce_block<2>(au, red);
        if (threadIdx.x == 0) {
            a.part[(size_t)1 * G + blockIdx.x] = au[0];
            a.part[(size_t)2 * G + blockIdx.x] = au[1];
        }
        if (!grid_barrier(a.bar, a.err, a.spin_limit)) {
            status = VX_TIMEOUT;
            break;
        }
        double tu[2];
        grid_totals<2>(a.part, G, su, red, tot, tu);
        its += 1;
        residual = sqrt(tu[1]) / initial;
        if (!isfinite(tu[0]) || !isfinite(tu[1])) {
            status = VX_NONFINITE;
            done = true;
        } else if (residual < a.tolerance) {
            done = true;
        } else if (its >= a.max_iterations) {
            status = VX_NOT_CONVERGED;
            done = true;
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        sc->iterations = its;
        sc->residual = residual;
        sc->initial = initial;
        sc->status = status;
        sc->done = 1;
    }
}

template <int R>
cudaError_t launch_r(const PersistArgs& a, unsigned G, size_t smem, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_pcg_persistent<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    PersistArgs args = a;
    void* params[] = {&args};
    return cudaLaunchCooperativeKernel((void*)k_pcg_persistent<R>, dim3(G), dim3(kPThreads), params, smem, st);
}

}  // namespace

// Whether the persistent inner solve fits this scene on this GPU; caches the shape.
bool persistent_plan(vx_scene* s) {
    if (s->persist_checked) return s->persist_ok;
    s->persist_checked = true;
    s->persist_ok = false;
    if (s->n == 0) return false;
    int dev = s->device, max_smem = 0, coop = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return false;
    unsigned G = (unsigned)s->sm_count;
    unsigned min_blocks = (s->n + 255) / 256;  // at least 256 REVs per block
    if (min_blocks < G) G = min_blocks;
    if (G == 0) G = 1;
    unsigned cap = (s->n + G - 1) / G;
    unsigned R = (cap + kPThreads - 1) / kPThreads;
    size_t smem = (size_t)kFloatsPerRev * cap * sizeof(float);
    if (R > 4 || smem + 4096 > (size_t)max_smem) return false;
    s->persist_G = G;
    s->persist_cap = cap;
    s->persist_R = R <= 1 ? 1 : (R <= 2 ? 2 : 4);
    s->persist_smem = smem;
    s->persist_ok = true;
    return true;
}

// One FP32 inner solve A32 d = r64 / |r64| in a single cooperative launch.
int32_t solve_inner_persistent(vx_scene* s, double tolerance, uint32_t max_iterations) {
    PersistArgs a;
    a.n = s->n;
    a.cap = s->persist_cap;
    a.flags = s->flags;
    a.D = s->d32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.nbr = s->nbr;
    a.rev = s->rev;
    a.src = s->r64;
    a.scale_from = &s->sc->r64_norm;
    a.x = s->x32;
    a.zg = s->z32;
    a.pg = s->p32[0];
    a.part = s->partials;
    a.bar = s->barrier;
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = s->sc32;
    a.tolerance = tolerance;
    a.max_iterations = max_iterations;
    a.spin_limit = 20000000ull;  // ~1-2 s of waiting at one barrier
    // VXCOROT_BARRIER_SPINS lowers the bound so a test can make the wait run out
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) {
        switch (s->persist_R) {
            case 1: e = launch_r<1>(a, s->persist_G, s->persist_smem, s->stream); break;
            case 2: e = launch_r<2>(a, s->persist_G, s->persist_smem, s->stream); break;
            default: e = launch_r<4>(a, s->persist_G, s->persist_smem, s->stream); break;
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
