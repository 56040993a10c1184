// vx_pcg.cu — block-Jacobi PCG on the assembly-free bond-lattice operator.
//
// Follows the CPU PCG of solve_coupled (src/solver.rs:1833-1911): x0 = 0,
// z = M^-1 r, p = z; alpha = rz / p.Ap (stop when p.Ap <= 1e-30); x += alpha p,
// r -= alpha Ap; stop when |r|/|r0| < tolerance (checked every iteration);
// z = M^-1 r; beta = r.z'/r.z; p = z + beta p. Dots accumulate in FP64; in the
// FP32 form alpha and beta are rounded to f32 as the reference does
// (src/solver.rs:1867, :1900).
//
// One iteration is two grid-stride kernels sized to fill the GPU once:
//   k_matvec  p_new = z + beta p_old (ping-pong buffers, formed for the REV and,
//             on the fly, for its six neighbours) and Ap (apply_row: in FP64
//             D p - P sum K p_nbr, in FP32 the same operator built from m/h^2);
//             writes per-block partials of p.Ap.
//   k_update  x += alpha p, r -= alpha Ap, z = D^-1 r; writes per-block partials
//             of r.z and r.r.
// Each kernel starts by summing the previous kernel's partials in a fixed order
// in every block, so every block derives the same alpha, beta, convergence and
// iteration-cap decisions without an atomic ticket or a serial tail; block 0
// records them for the host. Every load of a REV's data is issued before any of
// it is used (neighbour indices are clamped instead of branched on), so a
// thread keeps its whole stencil in flight. A chunk of 16 iterations is
// captured once as a CUDA graph and replayed; kernels after the stop decision
// return at entry.
#include <cstring>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_layout.cuh"
#include "vx_reduce.cuh"
#include "vx_pcg_core.cuh"

namespace vx {

constexpr int kChunk = 16;  // iterations per captured graph (even: p buffers alternate)

// ---- kernels ----------------------------------------------------------------------------
// r = scale * src (src FP64), x = 0, z = D^-1 r, p_old = 0; the r.z and r.r
// partials go to pu; the last block to finish sets the solve's scalars.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_init(IterArgs<T> a, const double* __restrict__ src,
                                                   const double* __restrict__ scale_from, double tolerance,
                                                   uint32_t max_iterations) {
    const size_t n = a.n;
    const size_t stride = (size_t)gridDim.x * kThreads;
    double scale = 1.0;
    if (scale_from) {
        double rn = *scale_from;
        scale = rn > 0.0 ? 1.0 / rn : 1.0;
    }
    double v[2] = {0.0, 0.0};
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        V3<T> r = {(T)(src[i] * scale), (T)(src[n + i] * scale), (T)(src[2 * n + i] * scale)};
        V3<T> z = mul(load_sym(a.Dinv, n, i), r);
        store_v(a.r, n, i, r);
        store_v(a.z, n, i, z);
        store_v(a.x, n, i, V3<T>{T(0), T(0), T(0)});
        store_v(const_cast<T*>(a.p_old), n, i, V3<T>{T(0), T(0), T(0)});
        v[0] += dot_d(r, z);
        v[1] += dot_d(r, r);
    }
    if (grid_sum<2>(v, a.pu, &a.sc->counter[0]) && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        sc->rz[0] = v[0];
        sc->rz[1] = INFINITY;  // beta of the first iteration is rz0 / inf = 0
        sc->rr = v[1];
        sc->initial = sqrt(v[1]);
        sc->beta = 0.0;
        sc->alpha = 0.0;
        sc->pap = 0.0;
        sc->residual = 0.0;
        sc->tolerance = tolerance;
        sc->max_iterations = max_iterations;
        sc->iterations = 0;
        sc->status = VX_OK;
        const bool trivial = !(sc->initial > 1e-12);
        int32_t done = (trivial || max_iterations == 0) ? 1 : 0;
        if (!isfinite(v[1]) || !isfinite(v[0])) {
            done = 1;
            sc->status = VX_NONFINITE;
        } else if (!trivial && max_iterations == 0) {
            sc->status = VX_NOT_CONVERGED;
        }
        sc->done = done;
    }
}

// Iteration k (PAR = k & 1): convergence test of iteration k-1, beta, then
// p_new = z + beta p_old and Ap = A p_new with p.Ap partials.
// The PCG kernels are latency-bound gathers; MB 256-thread blocks per SM is
// the register budget the compiler must meet (MB 4: 64 registers a thread).
// Unbounded it picks 79 in k_matvec<float> and 126 in k_update<double>, which
// halves the loads in flight: on the 160^3 lattice the FP32 matvec runs 2.1x
// faster at MB 4. The autotuner (vx_scene_autotune) picks MB per scene.
template <typename T, int PAR, int MB>
__global__ void __launch_bounds__(kThreads, MB) k_matvec(IterArgs<T> a) {
    __shared__ int32_t s_done;
    const unsigned G = gridDim.x;
    if (threadIdx.x == 0) s_done = *(volatile int32_t*)&a.sc->done;
    double t[2];
    block_total<2>(a.pu, G, t);  // its barrier publishes s_done
    if (s_done) return;
    PcgScalars* sc = a.sc;
    const uint32_t its = sc->iterations;
    const double rz = t[0], rr = t[1];
    const double residual = sqrt(rr) / sc->initial;
    int stop = 0, status = VX_OK;
    if (its > 0) {
        if (!isfinite(rr) || !isfinite(rz)) {
            stop = 1;
            status = VX_NONFINITE;
        } else if (residual < sc->tolerance) {
            stop = 1;
        }
    }
    if (!stop && its >= sc->max_iterations) {
        stop = 1;
        status = VX_NOT_CONVERGED;
    }
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    if (stop) {
        if (leader) {
            sc->status = status;
            if (its > 0) sc->residual = residual;
            sc->rr = rr;
            sc->done = 1;
        }
        return;
    }
    const T beta = (T)(rz / sc->rz[PAR ^ 1]);
    if (leader) {
        sc->rz[PAR] = rz;
        sc->beta = (double)beta;
        sc->rr = rr;
        if (its > 0) sc->residual = residual;
    }
    const size_t n = a.n;
    const size_t stride = (size_t)G * kThreads;
    const T* __restrict__ z_in = a.z_in;
    const T* __restrict__ p_old = a.p_old;
    auto get = [&](uint32_t j) {
        return V3<T>{fma(beta, __ldg(p_old + j), __ldg(z_in + j)), fma(beta, __ldg(p_old + n + j), __ldg(z_in + n + j)),
                     fma(beta, __ldg(p_old + 2 * n + j), __ldg(z_in + 2 * n + j))};
    };
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        V3<T> pi = get((uint32_t)i);
        V3<T> y = apply_row<T>(a, (uint32_t)i, pi, get);
        store_v(a.p_new, n, i, pi);
        store_v(a.ap, n, i, y);
        acc += dot_d(pi, y);
    }
    double v[1] = {acc};
    block_partial<1>(v, a.pm, G);
}

// Iteration k: alpha = rz_k / p.Ap, x += alpha p, r -= alpha Ap, z = D^-1 r with
// r.z and r.r partials; p.Ap <= 1e-30 stops like the reference (src/solver.rs:1864-1866).
template <typename T, int PAR, int MB>
__global__ void __launch_bounds__(kThreads, MB) k_update(IterArgs<T> a) {
    __shared__ int32_t s_done;
    const unsigned G = gridDim.x;
    if (threadIdx.x == 0) s_done = *(volatile int32_t*)&a.sc->done;
    double t[1];
    block_total<1>(a.pm, G, t);
    if (s_done) return;
    PcgScalars* sc = a.sc;
    const double pap = t[0];
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    if (!isfinite(pap) || pap <= 1e-30) {
        if (leader) {
            sc->pap = pap;
            sc->iterations += 1;
            if (!isfinite(pap)) sc->status = VX_NONFINITE;
            sc->done = 1;
        }
        return;
    }
    const T alpha = (T)(sc->rz[PAR] / pap);
    if (leader) {
        sc->pap = pap;
        sc->alpha = (double)alpha;
        sc->iterations += 1;
    }
    const size_t n = a.n;
    const size_t stride = (size_t)G * kThreads;
    double v[2] = {0.0, 0.0};
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        V3<T> p = ldg_v(a.p_new, n, i);
        V3<T> ap = ldg_v(a.ap, n, i);
        V3<T> x = load_v(a.x, n, i);
        V3<T> r = load_v(a.r, n, i);
        Sym<T> M = load_sym(a.Dinv, n, i);
        x = {fma(alpha, p.x, x.x), fma(alpha, p.y, x.y), fma(alpha, p.z, x.z)};
        r = {fma(-alpha, ap.x, r.x), fma(-alpha, ap.y, r.y), fma(-alpha, ap.z, r.z)};
        V3<T> z = mul(M, r);
        store_v(a.x, n, i, x);
        store_v(a.r, n, i, r);
        store_v(a.z, n, i, z);
        v[0] += dot_d(r, z);
        v[1] += dot_d(r, r);
    }
    block_partial<2>(v, a.pu, G);
}

// r64 = b - A64 x64 with |r64| and |b|; residual = |r64| / |b| (last-block finalize).
__global__ void __launch_bounds__(kThreads) k_residual64(IterArgs<double> a, const double* __restrict__ b,
                                                         double* __restrict__ r_out, PcgScalars* sc) {
    const size_t n = a.n;
    const size_t stride = (size_t)gridDim.x * kThreads;
    const double* x = a.x;
    auto get = [&](uint32_t j) { return V3<double>{x[j], x[n + j], x[2 * n + j]}; };
    double v[2] = {0.0, 0.0};
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        V3<double> y = apply_row<double>(a, (uint32_t)i, get((uint32_t)i), get);
        V3<double> bb = load_v(b, n, i);
        V3<double> r = {bb.x - y.x, bb.y - y.y, bb.z - y.z};
        store_v(r_out, n, i, r);
        v[0] += r.x * r.x + r.y * r.y + r.z * r.z;
        v[1] += bb.x * bb.x + bb.y * bb.y + bb.z * bb.z;
    }
    if (grid_sum<2>(v, a.pu, &sc->counter[3]) && threadIdx.x == 0) {
        sc->r64_norm = sqrt(v[0]);
        sc->b_norm = sqrt(v[1]);
        sc->residual = sc->b_norm > 0.0 ? sc->r64_norm / sc->b_norm : 0.0;
    }
}

// x64 += scale * x32 (inner correction back to the FP64 solution)
__global__ void k_accumulate(uint32_t n, double* __restrict__ x64, const float* __restrict__ x32,
                             const double* __restrict__ scale_from) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < 3 * (size_t)n) x64[t] += (*scale_from) * (double)x32[t];
}

// ---- drivers ------------------------------------------------------------------------------
static IterArgs<double> args64(vx_scene* s, int ping) {
    IterArgs<double> a{};
    a.n = s->n;
    a.kn = s->n;
    a.flags = s->flags;
    a.D = s->d64;
    a.K = s->bonds.k64;
    a.Dinv = s->dinv64;
    a.nbr = s->nbr;
    a.rev = s->rev;
    a.z_in = s->z64;
    a.p_old = s->p64[ping];
    a.p_new = s->p64[ping ^ 1];
    a.ap = s->ap64;
    a.x = s->x64;
    a.r = s->r64;
    a.z = s->z64;
    a.pm = s->partials;
    a.pu = s->partials + s->blocks;
    a.sc = s->sc;
    return a;
}

static IterArgs<float> args32(vx_scene* s, int ping) {
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
    a.pm = s->partials;
    a.pu = s->partials + s->blocks;
    a.sc = s->sc32;
    return a;
}

// The instantiations of the streaming kernels for one register budget.
template <typename T>
struct StreamKernels {
    void (*matvec[2])(IterArgs<T>);
    void (*update[2])(IterArgs<T>);
};
template <typename T>
static StreamKernels<T> stream_kernels(int mb) {
    switch (mb) {
        case 3: return {{k_matvec<T, 0, 3>, k_matvec<T, 1, 3>}, {k_update<T, 0, 3>, k_update<T, 1, 3>}};
        case 5: return {{k_matvec<T, 0, 5>, k_matvec<T, 1, 5>}, {k_update<T, 0, 5>, k_update<T, 1, 5>}};
        default: return {{k_matvec<T, 0, 4>, k_matvec<T, 1, 4>}, {k_update<T, 0, 4>, k_update<T, 1, 4>}};
    }
}

// Grid of the PCG kernels: enough blocks to fill every SM once, never more
// than there are 256-REV tiles.
template <typename T>
static unsigned pcg_grid(vx_scene* s) {
    unsigned* cached = sizeof(T) == 8 ? &s->grid64 : &s->grid32;
    if (*cached) return *cached;
    const StreamKernels<T> k = stream_kernels<T>(s->pcg_minb);
    int occ_m = 0, occ_u = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k.matvec[0], kThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, k.update[0], kThreads, 0);
    int occ = occ_m < occ_u ? occ_m : occ_u;
    if (occ < 1) occ = 1;
    unsigned g = (unsigned)(s->sm_count * occ);
    unsigned tiles = s->blocks ? s->blocks : 1;
    *cached = g < tiles ? g : tiles;
    return *cached;
}

template <typename T>
static void enqueue_chunk(vx_scene* s, cudaStream_t st) {
    const unsigned G = pcg_grid<T>(s);
    for (int it = 0; it < kChunk; it += 2) {
        IterArgs<T> a0, a1;
        if constexpr (sizeof(T) == 8) {
            a0 = args64(s, 0);
            a1 = args64(s, 1);
        } else {
            a0 = args32(s, 0);
            a1 = args32(s, 1);
        }
        const StreamKernels<T> k = stream_kernels<T>(s->pcg_minb);
        k.matvec[0]<<<G, kThreads, 0, st>>>(a0);
        k.update[0]<<<G, kThreads, 0, st>>>(a0);
        k.matvec[1]<<<G, kThreads, 0, st>>>(a1);
        k.update[1]<<<G, kThreads, 0, st>>>(a1);
    }
}

template <typename T>
static cudaError_t chunk_graph(vx_scene* s, cudaGraphExec_t* out) {
    if (*out) return cudaSuccess;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    enqueue_chunk<T>(s, s->stream);
    e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return e;
}

// Replays iteration chunks until the device reports done; one chunk stays in
// flight ahead of the host's check of the previous one. The device stops at
// the iteration cap, so at most cap/16 + 2 chunks run.
template <typename T>
static int32_t run_chunks(vx_scene* s, PcgScalars* sc, uint32_t max_iterations) {
    cudaGraphExec_t* g = sizeof(T) == 8 ? &s->chunk64 : &s->chunk32;
    cudaError_t e = chunk_graph<T>(s, g);
    if (e != cudaSuccess) {
        set_error("PCG graph capture failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    const uint32_t chunks = max_iterations / kChunk + 2;
    bool seen_done = false;
    for (uint32_t c = 0; c < chunks && !seen_done; ++c) {
        e = cudaGraphLaunch(*g, s->stream);
        s->launches += 2 * kChunk;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&s->h_done[c & 1], &sc->done, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaEventRecord(s->ev[c & 1], s->stream);
        if (e != cudaSuccess) {
            set_error("PCG chunk launch failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        if (c >= 1) {
            e = cudaEventSynchronize(s->ev[(c - 1) & 1]);
            if (e != cudaSuccess) {
                set_error("PCG chunk failed: %s", cudaGetErrorString(e));
                return VX_CUDA_ERROR;
            }
            seen_done = s->h_done[(c - 1) & 1] != 0;
        }
    }
    return VX_OK;
}

static int32_t fetch_scalars(vx_scene* s, PcgScalars* sc) {
    cudaError_t e = cudaMemcpyAsync(s->h_sc, sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        set_error("PCG scalar read failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

int32_t true_residual(vx_scene* s, double* out) {
    if (s->n == 0) {
        *out = 0.0;
        return VX_OK;
    }
    IterArgs<double> a = args64(s, 0);
    k_residual64<<<pcg_grid<double>(s), kThreads, 0, s->stream>>>(a, s->b64, s->r64, s->sc);
    int32_t st = fetch_scalars(s, s->sc);
    if (st != VX_OK) return st;
    *out = s->h_sc->residual;
    return VX_OK;
}

int32_t solve_fp64(vx_scene* s, double tolerance, uint32_t max_iterations, vx_pass_stats* out) {
    if (s->n == 0) {
        out->iterations = 0;
        out->residual = 0.0;
        out->converged = 1;
        return VX_OK;
    }
    IterArgs<double> a = args64(s, 0);
    k_init<double><<<pcg_grid<double>(s), kThreads, 0, s->stream>>>(a, s->b64, nullptr, tolerance, max_iterations);
    s->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("PCG init launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    int32_t st = run_chunks<double>(s, s->sc, max_iterations);
    if (st != VX_OK) return st;
    st = fetch_scalars(s, s->sc);
    if (st != VX_OK) return st;
    PcgScalars h = *s->h_sc;
    out->iterations = h.iterations;
    out->outer_iterations = 1;
    out->residual = h.residual;
    out->converged = h.status == VX_OK ? 1 : 0;
    return h.status;
}

int32_t solve_mixed(vx_scene* s, double tolerance, uint32_t max_iterations, double inner_tolerance,
                    uint32_t max_outer, int32_t kernel, vx_pass_stats* out) {
    out->iterations = 0;
    out->outer_iterations = 0;
    out->residual = 0.0;
    out->converged = 0;
    if (s->n == 0) {
        out->converged = 1;
        return VX_OK;
    }
    if (inner_tolerance <= 0.0) inner_tolerance = 1e-5;
    if (max_outer == 0) max_outer = 30;
    cudaMemsetAsync(s->x64, 0, 3 * (size_t)s->n * sizeof(double), s->stream);
    uint32_t used = 0;
    int32_t status = VX_NOT_CONVERGED;
    const unsigned G64 = pcg_grid<double>(s);
    const unsigned G32 = pcg_grid<float>(s);
    bool persistent = false;
    if (kernel == VX_KERNEL_PERSISTENT || (kernel == VX_KERNEL_AUTO && s->tuned_kernel != VX_KERNEL_STREAMING))
        persistent = persistent_plan(s);
    if (kernel == VX_KERNEL_PERSISTENT && !persistent) {
        set_error("the persistent inner solve does not fit this scene on this GPU");
        return VX_BAD_INPUT;
    }
    for (uint32_t outer = 0;; ++outer) {
        IterArgs<double> a64 = args64(s, 0);
        k_residual64<<<G64, kThreads, 0, s->stream>>>(a64, s->b64, s->r64, s->sc);
        s->launches += 1;
        int32_t st = fetch_scalars(s, s->sc);
        if (st != VX_OK) return st;
        PcgScalars h = *s->h_sc;
        out->residual = h.residual;
        if (!isfinite(h.residual)) {
            status = VX_NONFINITE;
            break;
        }
        if (h.b_norm <= 1e-12 || h.residual <= tolerance) {
            status = VX_OK;
            break;
        }
        if (outer >= max_outer || used >= max_iterations) break;
        // the inner solve only has to close the gap to the target, but no
        // tighter than the FP32 operator allows
        double inner = fmax(inner_tolerance, 0.5 * tolerance / h.residual);
        uint32_t budget = max_iterations - used;
        if (persistent) {
            st = solve_inner_persistent(s, inner, budget);
        } else {
            IterArgs<float> a32 = args32(s, 0);
            k_init<float><<<G32, kThreads, 0, s->stream>>>(a32, s->r64, &s->sc->r64_norm, inner, budget);
            s->launches += 1;
            st = run_chunks<float>(s, s->sc32, budget);
        }
        if (st != VX_OK) return st;
        st = fetch_scalars(s, s->sc32);
        if (st != VX_OK) return st;
        used += s->h_sc->iterations;
        out->outer_iterations = outer + 1;
        if (s->h_sc->status == VX_NONFINITE) {
            status = VX_NONFINITE;
            break;
        }
        if (s->h_sc->status == VX_TIMEOUT) {
            set_error("persistent PCG: a grid barrier wait ran out");
            return VX_TIMEOUT;
        }
        size_t m = 3 * (size_t)s->n;
        k_accumulate<<<(unsigned)((m + 255) / 256), 256, 0, s->stream>>>(s->n, s->x64, s->x32, &s->sc->r64_norm);
        s->launches += 1;
    }
    out->iterations = used;
    out->converged = status == VX_OK ? 1 : 0;
    return status;
}

int32_t kernel_times(vx_scene* s, int32_t precision, uint32_t reps, void* flush, uint64_t flush_bytes,
                     double* out_us) {
    if (s->n == 0) {
        out_us[0] = out_us[1] = 0.0;
        return VX_OK;
    }
    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    double tm = 0.0, tu = 0.0;
    cudaError_t err = cudaSuccess;
    for (uint32_t r = 0; r < reps && err == cudaSuccess; ++r) {
        float a_ms = 0.f, b_ms = 0.f;
        if (precision == VX_PRECISION_FP64) {
            const unsigned G = pcg_grid<double>(s);
            IterArgs<double> a = args64(s, 0);
            k_init<double><<<G, kThreads, 0, s->stream>>>(a, s->b64, nullptr, 0.0, 0xFFFFFFFFu);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[0], s->stream);
            stream_kernels<double>(s->pcg_minb).matvec[0]<<<G, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[1], s->stream);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[2], s->stream);
            stream_kernels<double>(s->pcg_minb).update[0]<<<G, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[3], s->stream);
        } else {
            const unsigned G = pcg_grid<float>(s);
            IterArgs<float> a = args32(s, 0);
            k_init<float><<<G, kThreads, 0, s->stream>>>(a, s->b64, nullptr, 0.0, 0xFFFFFFFFu);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[0], s->stream);
            stream_kernels<float>(s->pcg_minb).matvec[0]<<<G, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[1], s->stream);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[2], s->stream);
            stream_kernels<float>(s->pcg_minb).update[0]<<<G, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[3], s->stream);
        }
        err = cudaEventSynchronize(ev[3]);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&a_ms, ev[0], ev[1]);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&b_ms, ev[2], ev[3]);
        tm += a_ms;
        tu += b_ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (err != cudaSuccess) {
        set_error("kernel timing failed: %s", cudaGetErrorString(err));
        return VX_CUDA_ERROR;
    }
    out_us[0] = 1000.0 * tm / reps;
    out_us[1] = 1000.0 * tu / reps;
    out_us[2] = out_us[3] = out_us[4] = 0.0;
    if (precision == VX_PRECISION_MIXED && persistent_plan(s)) {
        // one persistent inner solve of a fixed iteration count on r = b
        const uint32_t iters = 64;
        cudaMemsetAsync(s->x64, 0, 3 * (size_t)s->n * sizeof(double), s->stream);
        IterArgs<double> a64 = args64(s, 0);
        k_residual64<<<pcg_grid<double>(s), kThreads, 0, s->stream>>>(a64, s->b64, s->r64, s->sc);
        if (flush_bytes) cudaMemsetAsync(flush, 0x5a, flush_bytes, s->stream);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s->stream);
        int32_t st = solve_inner_persistent(s, 0.0, iters);
        cudaEventRecord(e1, s->stream);
        float ms = 0.f;
        err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        int32_t its = 0;
        if (err == cudaSuccess) err = cudaMemcpy(&its, &s->sc32->iterations, 4, cudaMemcpyDeviceToHost);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != VX_OK) return st;
        if (err != cudaSuccess) {
            set_error("kernel timing failed: %s", cudaGetErrorString(err));
            return VX_CUDA_ERROR;
        }
        out_us[2] = its > 0 ? 1000.0 * ms / its : 0.0;
        out_us[3] = its;
        out_us[4] = s->exp_ok ? 3.0 : (s->brick_ok ? 1.0 : 2.0);
    }
    return VX_OK;
}


// ---- autotuning ------------------------------------------------------------------------
// Selects the register budget of the streaming kernels; the cached graphs
// and grids of the old budget are dropped.
static void set_minb(vx_scene* s, int mb) {
    if (s->pcg_minb == mb) return;
    cudaStreamSynchronize(s->stream);
    if (s->chunk64) cudaGraphExecDestroy(s->chunk64);
    if (s->chunk32) cudaGraphExecDestroy(s->chunk32);
    s->chunk64 = s->chunk32 = nullptr;
    s->grid64 = s->grid32 = 0;
    s->pcg_minb = mb;
}

// Microseconds per iteration of a 64-iteration inner solve from r = b
// (tolerance 0, so every iteration runs), CUDA events on the scene stream;
// the first run of a candidate warms its graph and is not timed.
int32_t time_candidate(vx_scene* s, int32_t precision, int32_t kernel, int mb, double* us) {
    const uint32_t iters = 64;
    if (kernel == VX_KERNEL_PERSISTENT) {
        s->persist_form = mb;  // mb names the persistent form (VX_PERSIST_*)
        s->persist_checked = false;
        if (!persistent_plan(s)) {
            *us = 1e30;
            return VX_OK;
        }
    } else {
        set_minb(s, mb);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0.f;
    uint32_t its = 0;
    int32_t st = VX_OK;
    cudaError_t err = cudaSuccess;
    for (int rep = 0; rep < 2 && st == VX_OK && err == cudaSuccess; ++rep) {
        PcgScalars* sc = precision == VX_PRECISION_FP64 ? s->sc : s->sc32;
        if (precision == VX_PRECISION_MIXED) {
            cudaMemsetAsync(s->x64, 0, 3 * (size_t)s->n * sizeof(double), s->stream);
            IterArgs<double> a64 = args64(s, 0);
            k_residual64<<<pcg_grid<double>(s), kThreads, 0, s->stream>>>(a64, s->b64, s->r64, s->sc);
        }
        cudaEventRecord(e0, s->stream);
        if (precision == VX_PRECISION_FP64) {
            IterArgs<double> a = args64(s, 0);
            k_init<double><<<pcg_grid<double>(s), kThreads, 0, s->stream>>>(a, s->b64, nullptr, 0.0, iters);
            st = run_chunks<double>(s, sc, iters);
        } else if (kernel == VX_KERNEL_PERSISTENT) {
            st = solve_inner_persistent(s, 0.0, iters);
        } else {
            IterArgs<float> a = args32(s, 0);
            k_init<float><<<pcg_grid<float>(s), kThreads, 0, s->stream>>>(a, s->r64, &s->sc->r64_norm, 0.0, iters);
            st = run_chunks<float>(s, sc, iters);
        }
        cudaEventRecord(e1, s->stream);
        err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess) err = cudaMemcpy(&its, &sc->iterations, 4, cudaMemcpyDeviceToHost);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != VX_OK) return st;
    if (err != cudaSuccess) {
        set_error("autotune timing failed: %s", cudaGetErrorString(err));
        return VX_CUDA_ERROR;
    }
    *us = its ? 1000.0 * ms / its : 1e30;
    return VX_OK;
}

// Streaming: mb is the register budget (blocks per SM). Persistent: mb is the
// form (VX_PERSIST_*), and the plan is rebuilt for it at the next pass.
void apply_tuning(vx_scene* s, int32_t kernel, int mb) {
    if (kernel == VX_KERNEL_PERSISTENT) {
        if (s->persist_form != mb) {
            s->persist_form = mb;
            s->persist_checked = false;
        }
    } else {
        set_minb(s, mb);
    }
    s->tuned_kernel = kernel;
}

}  // namespace vx
