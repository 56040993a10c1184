// vx_pcg.cu — block-Jacobi PCG on the assembly-free bond-lattice operator.
//
// Follows the CPU PCG of solve_coupled (src/solver.rs:1833-1911): x0 = 0,
// z = M^-1 r, p = z; alpha = rz / p.Ap (stop when p.Ap <= 1e-30); x += alpha p,
// r -= alpha Ap; stop when |r|/|r0| < tolerance (checked every iteration);
// z = M^-1 r; beta = r.z'/r.z; p = z + beta p. Dots accumulate in FP64.
//
// One iteration is two kernels:
//   k_matvec  p_new = z + beta p_old (ping-pong buffers, computed for the REV
//             and, on the fly, for its six neighbours), Ap = D p - P sum K p_nbr,
//             fused p.Ap grid reduction; its last block forms alpha.
//   k_update  x += alpha p, r -= alpha Ap, z = D^-1 r, fused r.z and r.r grid
//             reductions; its last block tests convergence and forms beta.
// Grid reductions are single-pass and deterministic: each block writes one
// partial, the last block to finish (atomic ticket) sums the partials in a
// fixed order. Kernels return at once when the device `done` flag is set, so
// a CUDA graph of a fixed chunk of iterations can be replayed until the host
// sees convergence.
#include <cstring>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_reduce.cuh"

namespace vx {

constexpr int kChunk = 16;  // iterations per captured graph (even: p buffers alternate)

template <typename T>
struct IterArgs {
    uint32_t n;
    const uint8_t* flags;
    const T* D;       // [6][n] projected diagonal
    const T* K;       // [18][n] bond K per axis (sym6), zero when not assembled
    const T* Dinv;    // [6][n]
    const uint32_t* nbr;
    const uint32_t* rev;
    const T* z_in;    // matvec: z
    const T* p_old;   // matvec: previous direction
    T* p_new;         // matvec: new direction
    T* ap;
    T* x;
    T* r;
    T* z;
    double* partials;
    PcgScalars* sc;
};

template <typename T>
__device__ __forceinline__ T round_scalar(double v) {
    return (T)v;
}

// ---- operator -------------------------------------------------------------------
template <typename T>
struct Vec3T {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ Vec3T<T> sym_mul(const T* S, size_t stride, size_t i, Vec3T<T> v) {
    T xx = S[i], yy = S[stride + i], zz = S[2 * stride + i];
    T xy = S[3 * stride + i], xz = S[4 * stride + i], yz = S[5 * stride + i];
    return {xx * v.x + xy * v.y + xz * v.z, xy * v.x + yy * v.y + yz * v.z, xz * v.x + yz * v.y + zz * v.z};
}

// A v at REV i: D_i v_i - P_i (sum over the three owned bonds K_(a,i) v_nbr
// + sum over the three bonds owned by the -axis neighbours K_(a,k) v_k).
// `fetch(j)` returns v_j. Neighbours with no free axis hold v = 0.
template <typename T, typename Fetch>
__device__ __forceinline__ Vec3T<T> apply_row(const IterArgs<T>& a, uint32_t i, Vec3T<T> vi, Fetch fetch) {
    const uint32_t n = a.n;
    Vec3T<T> y = sym_mul<T>(a.D, n, i, vi);
    Vec3T<T> s = {T(0), T(0), T(0)};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        uint32_t j = a.nbr[(size_t)ax * n + i];
        if (j != VX_EMPTY_U32) {
            Vec3T<T> kv = sym_mul<T>(a.K + (size_t)ax * 6 * n, n, i, fetch(j));
            s.x += kv.x;
            s.y += kv.y;
            s.z += kv.z;
        }
        uint32_t k = a.rev[(size_t)ax * n + i];
        if (k != VX_EMPTY_U32) {
            Vec3T<T> kv = sym_mul<T>(a.K + (size_t)ax * 6 * n, n, k, fetch(k));
            s.x += kv.x;
            s.y += kv.y;
            s.z += kv.z;
        }
    }
    uint8_t fl = a.flags[i];
    if (fl & 1) y.x -= s.x;
    if (fl & 2) y.y -= s.y;
    if (fl & 4) y.z -= s.z;
    return y;
}

// ---- kernels ----------------------------------------------------------------------
// r = scale * src (src FP64), x = 0, z = D^-1 r, p_old = 0; r.z and r.r.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_init(IterArgs<T> a, const double* __restrict__ src,
                                                   const double* __restrict__ scale_from, double tolerance,
                                                   uint32_t max_iterations) {
    const uint32_t n = a.n;
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    double scale = 1.0;
    if (scale_from) {
        double rn = *scale_from;
        scale = rn > 0.0 ? 1.0 / rn : 1.0;
    }
    double v[2] = {0.0, 0.0};
    if (i < n) {
        Vec3T<T> r = {(T)(src[i] * scale), (T)(src[n + i] * scale), (T)(src[2 * (size_t)n + i] * scale)};
        Vec3T<T> z = sym_mul<T>(a.Dinv, n, i, r);
        a.r[i] = r.x;
        a.r[n + i] = r.y;
        a.r[2 * (size_t)n + i] = r.z;
        a.z[i] = z.x;
        a.z[n + i] = z.y;
        a.z[2 * (size_t)n + i] = z.z;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a.x[(size_t)c * n + i] = T(0);
            const_cast<T*>(a.p_old)[(size_t)c * n + i] = T(0);
        }
        v[0] = (double)r.x * (double)z.x + (double)r.y * (double)z.y + (double)r.z * (double)z.z;
        v[1] = (double)r.x * (double)r.x + (double)r.y * (double)r.y + (double)r.z * (double)r.z;
    }
    if (grid_sum<2>(v, a.partials, &a.sc->counter[0]) && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        sc->rz = v[0];
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
        bool trivial = !(sc->initial > 1e-12);
        sc->done = (trivial || max_iterations == 0) ? 1 : 0;
        if (!isfinite(v[1]) || !isfinite(v[0])) {
            sc->done = 1;
            sc->status = VX_NONFINITE;
        } else if (!trivial && max_iterations == 0) {
            sc->status = VX_NOT_CONVERGED;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_matvec(IterArgs<T> a) {
    if (*(volatile int32_t*)&a.sc->done) return;
    const uint32_t n = a.n;
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const T beta = (T)a.sc->beta;
    double v[1] = {0.0};
    if (i < n) {
        auto fetch = [&](uint32_t j) {
            return Vec3T<T>{fma(beta, a.p_old[j], a.z_in[j]), fma(beta, a.p_old[n + j], a.z_in[n + j]),
                            fma(beta, a.p_old[2 * (size_t)n + j], a.z_in[2 * (size_t)n + j])};
        };
        Vec3T<T> pi = fetch(i);
        a.p_new[i] = pi.x;
        a.p_new[n + i] = pi.y;
        a.p_new[2 * (size_t)n + i] = pi.z;
        Vec3T<T> y = apply_row<T>(a, i, pi, fetch);
        a.ap[i] = y.x;
        a.ap[n + i] = y.y;
        a.ap[2 * (size_t)n + i] = y.z;
        v[0] = (double)pi.x * (double)y.x + (double)pi.y * (double)y.y + (double)pi.z * (double)y.z;
    }
    if (grid_sum<1>(v, a.partials, &a.sc->counter[1]) && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        double pap = v[0];
        sc->pap = pap;
        sc->iterations += 1;
        if (!isfinite(pap)) {
            sc->done = 1;
            sc->status = VX_NONFINITE;
        } else if (pap <= 1e-30) {
            sc->done = 1;  // breakdown: the reference stops without an error
        } else {
            sc->alpha = (double)round_scalar<T>(sc->rz / pap);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_update(IterArgs<T> a) {
    if (*(volatile int32_t*)&a.sc->done) return;
    const uint32_t n = a.n;
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const T alpha = (T)a.sc->alpha;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        Vec3T<T> r;
        T* rc[3] = {&r.x, &r.y, &r.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            size_t t = (size_t)c * n + i;
            T p = a.p_new[t];
            a.x[t] = fma(alpha, p, a.x[t]);
            *rc[c] = fma(-alpha, a.ap[t], a.r[t]);
            a.r[t] = *rc[c];
        }
        Vec3T<T> z = sym_mul<T>(a.Dinv, n, i, r);
        a.z[i] = z.x;
        a.z[n + i] = z.y;
        a.z[2 * (size_t)n + i] = z.z;
        v[0] = (double)r.x * (double)z.x + (double)r.y * (double)z.y + (double)r.z * (double)z.z;
        v[1] = (double)r.x * (double)r.x + (double)r.y * (double)r.y + (double)r.z * (double)r.z;
    }
    if (grid_sum<2>(v, a.partials, &a.sc->counter[2]) && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        double rz_new = v[0], rr = v[1];
        sc->rr = rr;
        double residual = sqrt(rr) / sc->initial;
        sc->residual = residual;
        if (!isfinite(rr) || !isfinite(rz_new)) {
            sc->done = 1;
            sc->status = VX_NONFINITE;
        } else if (residual < sc->tolerance) {
            sc->done = 1;
            sc->status = VX_OK;
        } else if (sc->iterations >= sc->max_iterations) {
            sc->done = 1;
            sc->status = VX_NOT_CONVERGED;
        } else {
            sc->beta = (double)round_scalar<T>(rz_new / sc->rz);
            sc->rz = rz_new;
        }
    }
}

// r64 = b - A64 x64 with |r64| and |b|; residual = |r64| / |b|.
__global__ void __launch_bounds__(kThreads) k_residual64(IterArgs<double> a, const double* __restrict__ b,
                                                         double* __restrict__ r_out, PcgScalars* sc) {
    const uint32_t n = a.n;
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        const double* x = a.x;
        auto fetch = [&](uint32_t j) { return Vec3T<double>{x[j], x[n + j], x[2 * (size_t)n + j]}; };
        Vec3T<double> y = apply_row<double>(a, i, fetch(i), fetch);
        double bx = b[i], by = b[n + i], bz = b[2 * (size_t)n + i];
        double rx = bx - y.x, ry = by - y.y, rz = bz - y.z;
        r_out[i] = rx;
        r_out[n + i] = ry;
        r_out[2 * (size_t)n + i] = rz;
        v[0] = rx * rx + ry * ry + rz * rz;
        v[1] = bx * bx + by * by + bz * bz;
    }
    if (grid_sum<2>(v, a.partials, &sc->counter[3]) && threadIdx.x == 0) {
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

// ---- drivers ------------------------------------------------------------------------
static IterArgs<double> args64(vx_scene* s, int ping) {
    IterArgs<double> a;
    a.n = s->n;
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
    a.partials = s->partials;
    a.sc = s->sc;
    return a;
}

static IterArgs<float> args32(vx_scene* s, int ping) {
    IterArgs<float> a;
    a.n = s->n;
    a.flags = s->flags;
    a.D = s->d32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.nbr = s->nbr;
    a.rev = s->rev;
    a.z_in = s->z32;
    a.p_old = s->p32[ping];
    a.p_new = s->p32[ping ^ 1];
    a.ap = s->ap32;
    a.x = s->x32;
    a.r = s->r32;
    a.z = s->z32;
    a.partials = s->partials;
    a.sc = s->sc32;
    return a;
}

template <typename T>
static void enqueue_chunk(vx_scene* s, cudaStream_t st) {
    for (int it = 0; it < kChunk; ++it) {
        int ping = it & 1;
        IterArgs<T> a;
        if constexpr (sizeof(T) == 8) a = args64(s, ping);
        else a = args32(s, ping);
        k_matvec<T><<<s->blocks, kThreads, 0, st>>>(a);
        // the update reads the new direction
        k_update<T><<<s->blocks, kThreads, 0, st>>>(a);
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
// flight ahead of the host's check of the previous one.
template <typename T>
static int32_t run_chunks(vx_scene* s, PcgScalars* sc, uint32_t max_iterations) {
    cudaGraphExec_t* g = sizeof(T) == 8 ? &s->chunk64 : &s->chunk32;
    cudaError_t e = chunk_graph<T>(s, g);
    if (e != cudaSuccess) {
        set_error("PCG graph capture failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    uint32_t chunks = (max_iterations + kChunk - 1) / kChunk;
    for (uint32_t c = 0; c < chunks; ++c) {
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
            if (s->h_done[(c - 1) & 1]) break;
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
    k_residual64<<<s->blocks, kThreads, 0, s->stream>>>(a, s->b64, s->r64, s->sc);
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
    k_init<double><<<s->blocks, kThreads, 0, s->stream>>>(a, s->b64, nullptr, tolerance, max_iterations);
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
                    uint32_t max_outer, vx_pass_stats* out) {
    out->iterations = 0;
    out->outer_iterations = 0;
    out->residual = 0.0;
    out->converged = 0;
    if (s->n == 0) {
        out->converged = 1;
        return VX_OK;
    }
    if (inner_tolerance <= 0.0) inner_tolerance = 1e-4;
    if (max_outer == 0) max_outer = 30;
    cudaMemsetAsync(s->x64, 0, 3 * (size_t)s->n * sizeof(double), s->stream);
    uint32_t used = 0;
    int32_t status = VX_NOT_CONVERGED;
    for (uint32_t outer = 0;; ++outer) {
        IterArgs<double> a64 = args64(s, 0);
        k_residual64<<<s->blocks, kThreads, 0, s->stream>>>(a64, s->b64, s->r64, s->sc);
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
        IterArgs<float> a32 = args32(s, 0);
        k_init<float><<<s->blocks, kThreads, 0, s->stream>>>(a32, s->r64, &s->sc->r64_norm, inner, budget);
        s->launches += 1;
        st = run_chunks<float>(s, s->sc32, budget);
        if (st != VX_OK) return st;
        st = fetch_scalars(s, s->sc32);
        if (st != VX_OK) return st;
        used += s->h_sc->iterations;
        out->outer_iterations = outer + 1;
        if (s->h_sc->status == VX_NONFINITE) {
            status = VX_NONFINITE;
            break;
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
            IterArgs<double> a = args64(s, 0);
            k_init<double><<<s->blocks, kThreads, 0, s->stream>>>(a, s->b64, nullptr, 0.0, 0xFFFFFFFFu);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[0], s->stream);
            k_matvec<double><<<s->blocks, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[1], s->stream);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[2], s->stream);
            k_update<double><<<s->blocks, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[3], s->stream);
        } else {
            IterArgs<float> a = args32(s, 0);
            k_init<float><<<s->blocks, kThreads, 0, s->stream>>>(a, s->b64, nullptr, 0.0, 0xFFFFFFFFu);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[0], s->stream);
            k_matvec<float><<<s->blocks, kThreads, 0, s->stream>>>(a);
            cudaEventRecord(ev[1], s->stream);
            if (flush_bytes) cudaMemsetAsync(flush, (int)(r & 0xff), flush_bytes, s->stream);
            cudaEventRecord(ev[2], s->stream);
            k_update<float><<<s->blocks, kThreads, 0, s->stream>>>(a);
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
    return VX_OK;
}

}  // namespace vx
