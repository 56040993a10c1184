// vx_shim.cu — vx_solve_pcg_f32, the drop-in for cuda_solver::solve_pcg.
//
// Same inputs, layouts and convergence rule as src/cuda_solver.rs:301-501 with
// the arithmetic of the kernels in src/cuda/pcg.ptx (f32 vectors, f32 fused
// multiply-adds in the same order, f64 dot accumulation, f32 alpha/beta with
// the 1e-30 guards). Differences are in how the work is scheduled: the
// direction update is fused into the next matvec, the three dots of an
// iteration are fused into the matvec and update kernels as multi-block
// reductions instead of single-CTA loops, and 16 iterations are replayed as
// one CUDA graph between the host's residual checks (the reference checks
// every 16 iterations too).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "vx_internal.h"
#include "vx_reduce.cuh"

namespace vx {
namespace {

struct ShimScalars {
    double rho;    // r . z
    double pap;
    double rr;
    double alpha;  // f32 value
    double beta;   // f32 value
    uint32_t counter[3];
};

struct ShimArgs {
    uint32_t n;
    const uint32_t* nbr6;
    const float* diag9;
    const float* blocks54;
    const float* inv9;
    const float* z_in;
    const float* p_old;
    float* p_new;
    float* ap;
    float* dx;
    float* r;
    float* z;
    double* partials;
    ShimScalars* sc;
};

// out_r = m_r0 v0 (mul), then fma m_r1 v1, fma m_r2 v2 (pcg.ptx:39-47)
__device__ __forceinline__ void m3v(const float* m, const float* v, float* o) {
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = fmaf(m[3 * r + 2], v[2], fmaf(m[3 * r + 1], v[1], m[3 * r] * v[0]));
}
__device__ __forceinline__ double dot_ptx(const float* a, const float* b) {
    double v = (double)a[0] * (double)b[0];
    v = fma((double)a[1], (double)b[1], v);
    return fma((double)a[2], (double)b[2], v);
}

__global__ void __launch_bounds__(kThreads) k_shim_init(ShimArgs a) {
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    double v[1] = {0.0};
    if (i < a.n) {
        float r[3] = {a.r[3 * (size_t)i], a.r[3 * (size_t)i + 1], a.r[3 * (size_t)i + 2]};
        float z[3];
        m3v(a.inv9 + 9 * (size_t)i, r, z);
        for (int c = 0; c < 3; ++c) {
            a.z[3 * (size_t)i + c] = z[c];
            a.dx[3 * (size_t)i + c] = 0.0f;
            const_cast<float*>(a.p_old)[3 * (size_t)i + c] = 0.0f;
        }
        v[0] = dot_ptx(r, z);
    }
    if (grid_sum<1>(v, a.partials, &a.sc->counter[0]) && threadIdx.x == 0) {
        a.sc->rho = v[0];
        a.sc->beta = 0.0;
    }
}

// p_new = beta p_old + z; Ap = D p + sum_s B_s p_nbr(s) (pcg.ptx:4-103, :199-230);
// alpha = f32(rho / p.Ap), or 0 when p.Ap <= 1e-30 (:639-724)
__global__ void __launch_bounds__(kThreads) k_shim_matvec(ShimArgs a) {
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const float beta = (float)a.sc->beta;
    double v[1] = {0.0};
    if (i < a.n) {
        float p[3];
        for (int c = 0; c < 3; ++c) {
            p[c] = fmaf(beta, a.p_old[3 * (size_t)i + c], a.z_in[3 * (size_t)i + c]);
            a.p_new[3 * (size_t)i + c] = p[c];
        }
        float acc[3];
        m3v(a.diag9 + 9 * (size_t)i, p, acc);
        for (int s = 0; s < 6; ++s) {
            uint32_t j = a.nbr6[6 * (size_t)i + s];
            if (j == VX_EMPTY_U32) continue;
            float x[3];
            for (int c = 0; c < 3; ++c) x[c] = fmaf(beta, a.p_old[3 * (size_t)j + c], a.z_in[3 * (size_t)j + c]);
            const float* b = a.blocks54 + 54 * (size_t)i + 9 * s;
            for (int r = 0; r < 3; ++r) {
                acc[r] = fmaf(b[3 * r], x[0], acc[r]);
                acc[r] = fmaf(b[3 * r + 1], x[1], acc[r]);
                acc[r] = fmaf(b[3 * r + 2], x[2], acc[r]);
            }
        }
        for (int c = 0; c < 3; ++c) a.ap[3 * (size_t)i + c] = acc[c];
        v[0] = dot_ptx(p, acc);
    }
    if (grid_sum<1>(v, a.partials, &a.sc->counter[1]) && threadIdx.x == 0) {
        double den = v[0];
        a.sc->pap = den;
        a.sc->alpha = den > 1e-30 ? (double)(float)(a.sc->rho / den) : 0.0;
    }
}

// dx += alpha p; r -= alpha Ap; z = inverse r (pcg.ptx:468-557); rho' = r.z,
// beta = f32(rho'/rho) or 0 when rho <= 1e-30 (:437-466); r.r for the checkpoint.
__global__ void __launch_bounds__(kThreads) k_shim_update(ShimArgs a) {
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const float alpha = (float)a.sc->alpha;
    double v[2] = {0.0, 0.0};
    if (i < a.n) {
        float r[3], z[3];
        for (int c = 0; c < 3; ++c) {
            size_t t = 3 * (size_t)i + c;
            a.dx[t] = fmaf(alpha, a.p_new[t], a.dx[t]);
            r[c] = fmaf(-alpha, a.ap[t], a.r[t]);
            a.r[t] = r[c];
        }
        m3v(a.inv9 + 9 * (size_t)i, r, z);
        for (int c = 0; c < 3; ++c) a.z[3 * (size_t)i + c] = z[c];
        v[0] = dot_ptx(r, z);
        v[1] = dot_ptx(r, r);
    }
    if (grid_sum<2>(v, a.partials, &a.sc->counter[2]) && threadIdx.x == 0) {
        double rho = a.sc->rho;
        a.sc->beta = rho > 1e-30 ? (double)(float)(v[0] / rho) : 0.0;
        a.sc->rho = v[0];
        a.sc->rr = v[1];
    }
}

// Process-wide solver state with grow-only buffers, like the reference's
// OnceLock<Mutex<CudaSolver>> (src/cuda_solver.rs:66, :162-181).
struct Shim {
    std::mutex lock;
    bool init = false;
    cudaStream_t stream = nullptr;
    char* buf = nullptr;
    size_t cap = 0;
    ShimScalars* h_sc = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_n = 0;
    char* graph_buf = nullptr;
};
Shim g_shim;

constexpr int kShimChunk = 16;

// Puts the caller's current device back when the shim returns: the shim works
// on device 0 (as cuda_solver.rs does) and must not move the calling thread.
struct DeviceRestore {
    int device = -1;
    DeviceRestore() {
        if (cudaGetDevice(&device) != cudaSuccess) {
            device = -1;
            (void)cudaGetLastError();
        }
    }
    ~DeviceRestore() {
        if (device >= 0) cudaSetDevice(device);
    }
};

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" int32_t vx_solve_pcg_f32(const float* rhs, const uint32_t* neighbors, const float* diagonal,
                                    const float* blocks, const float* inverse_diagonal, uint32_t n,
                                    uint32_t max_iterations, float tolerance, float* out_dx,
                                    uint32_t* out_iterations, float* out_relative) {
    clear_error();
    if (out_iterations) *out_iterations = 0;
    if (out_relative) *out_relative = 0.0f;
    if (n == 0) return VX_OK;
    if (!rhs || !neighbors || !diagonal || !blocks || !inverse_diagonal || !out_dx) {
        set_error("vx_solve_pcg_f32: null argument");
        return VX_BAD_INPUT;
    }
    for (size_t e = 0; e < 6 * (size_t)n; ++e)
        if (neighbors[e] != VX_EMPTY && neighbors[e] >= n) {
            set_error("vx_solve_pcg_f32: neighbour slot %zu points at row %u of %u", e, neighbors[e], n);
            return VX_BAD_INPUT;
        }
    double initial_sq = 0.0;
    for (size_t t = 0; t < 3 * (size_t)n; ++t) initial_sq += (double)rhs[t] * (double)rhs[t];
    double initial = std::sqrt(initial_sq);
    if (initial <= 1e-12) {
        std::memset(out_dx, 0, 3 * (size_t)n * sizeof(float));
        return VX_OK;
    }
    std::lock_guard<std::mutex> guard(g_shim.lock);
    DeviceRestore restore;
    Shim& S = g_shim;
    cudaError_t e = cudaSuccess;
    if (!S.init) {
        int count = 0;
        e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0) {
            set_error("vx_solve_pcg_f32: no CUDA device (%s)", cudaGetErrorString(e));
            return VX_NO_DEVICE;
        }
        e = cudaSetDevice(0);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMallocHost(&S.h_sc, sizeof(ShimScalars));
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32: CUDA initialisation failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        S.init = true;
    }
    cudaSetDevice(0);
    size_t m = n;
    unsigned blocks_n = (unsigned)((m + kThreads - 1) / kThreads);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t off_nbr = 0, off_diag = off_nbr + al(6 * m * 4), off_blk = off_diag + al(9 * m * 4),
           off_inv = off_blk + al(54 * m * 4), off_r = off_inv + al(9 * m * 4), off_dx = off_r + al(3 * m * 4),
           off_z = off_dx + al(3 * m * 4), off_p0 = off_z + al(3 * m * 4), off_p1 = off_p0 + al(3 * m * 4),
           off_ap = off_p1 + al(3 * m * 4), off_part = off_ap + al(3 * m * 4),
           off_sc = off_part + al(2 * (size_t)blocks_n * 8), total = off_sc + al(sizeof(ShimScalars));
    if (total > S.cap) {
        if (S.graph) {
            cudaGraphExecDestroy(S.graph);
            S.graph = nullptr;
        }
        if (S.buf) cudaFree(S.buf);
        S.buf = nullptr;
        S.cap = 0;
        e = cudaMalloc(&S.buf, total);
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32: device allocation of %zu bytes failed: %s", total, cudaGetErrorString(e));
            return VX_OOM;
        }
        S.cap = total;
    }
    char* B = S.buf;
    ShimArgs A[2];
    for (int k = 0; k < 2; ++k) {
        A[k].n = n;
        A[k].nbr6 = (const uint32_t*)(B + off_nbr);
        A[k].diag9 = (const float*)(B + off_diag);
        A[k].blocks54 = (const float*)(B + off_blk);
        A[k].inv9 = (const float*)(B + off_inv);
        A[k].z_in = (const float*)(B + off_z);
        A[k].p_old = (const float*)(B + (k ? off_p1 : off_p0));
        A[k].p_new = (float*)(B + (k ? off_p0 : off_p1));
        A[k].ap = (float*)(B + off_ap);
        A[k].dx = (float*)(B + off_dx);
        A[k].r = (float*)(B + off_r);
        A[k].z = (float*)(B + off_z);
        A[k].partials = (double*)(B + off_part);
        A[k].sc = (ShimScalars*)(B + off_sc);
    }
    cudaStream_t st = S.stream;
    // the matrix is uploaded on every call, as in the reference (src/cuda_solver.rs:337-364)
    e = cudaMemcpyAsync(B + off_nbr, neighbors, 6 * m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B + off_diag, diagonal, 9 * m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B + off_blk, blocks, 54 * m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B + off_inv, inverse_diagonal, 9 * m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B + off_r, rhs, 3 * m * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(B + off_sc, 0, sizeof(ShimScalars), st);
    if (e != cudaSuccess) {
        set_error("vx_solve_pcg_f32: upload failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    k_shim_init<<<blocks_n, kThreads, 0, st>>>(A[0]);
    // graph of 16 iterations for this size and buffer
    if (!S.graph || S.graph_n != n || S.graph_buf != S.buf) {
        if (S.graph) cudaGraphExecDestroy(S.graph);
        S.graph = nullptr;
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int it = 0; it < kShimChunk; ++it) {
                k_shim_matvec<<<blocks_n, kThreads, 0, st>>>(A[it & 1]);
                k_shim_update<<<blocks_n, kThreads, 0, st>>>(A[it & 1]);
            }
            e = cudaStreamEndCapture(st, &g);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&S.graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32: graph capture failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        S.graph_n = n;
        S.graph_buf = S.buf;
    }
    uint32_t it = 0;
    double rr = INFINITY;
    int ping = 0;
    while (it < max_iterations) {
        uint32_t todo = max_iterations - it;
        if (todo >= (uint32_t)kShimChunk && ping == 0) {
            e = cudaGraphLaunch(S.graph, st);
            it += kShimChunk;
        } else {
            uint32_t step = todo < (uint32_t)kShimChunk ? todo : (uint32_t)kShimChunk;
            for (uint32_t k = 0; k < step; ++k) {
                k_shim_matvec<<<blocks_n, kThreads, 0, st>>>(A[ping]);
                k_shim_update<<<blocks_n, kThreads, 0, st>>>(A[ping]);
                ping ^= 1;
            }
            it += step;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(S.h_sc, A[0].sc, sizeof(ShimScalars), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32: iteration failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        rr = S.h_sc->rr;
        if (!std::isfinite(rr) || rr < 0.0) break;
        float relative = (float)(std::sqrt(rr) / initial);
        if (relative <= tolerance) break;
    }
    // the final direction of an odd tail lives in the other buffer; dx is what is returned
    e = cudaMemcpyAsync(out_dx, B + off_dx, 3 * m * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error("vx_solve_pcg_f32: download failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    if (out_iterations) *out_iterations = it;
    if (!std::isfinite(rr) || rr < 0.0) {
        set_error("CUDA PCG produced a non-finite residual norm");
        return VX_NONFINITE;
    }
    float relative = (float)(std::sqrt(rr) / initial);
    if (out_relative) *out_relative = relative;
    if (!std::isfinite(relative) || relative > tolerance) {
        set_error("CUDA PCG did not converge: iterations=%u, relative residual=%.3e, tolerance=%.3e", it, relative,
                  tolerance);
        return VX_NOT_CONVERGED;
    }
    for (size_t t = 0; t < 3 * m; ++t)
        if (!std::isfinite(out_dx[t])) {
            set_error("CUDA PCG produced a non-finite correction");
            return VX_NONFINITE;
        }
    return VX_OK;
}

// ---------------------------------------------------------------------------
// vx_solve_pcg_f32_noalloc: the same block-Jacobi PCG as vx_solve_pcg_f32, for
// callers that cannot allocate device memory. Inputs and the output correction
// are caller-owned device buffers; the solver's own work vectors, reduction
// partials and scalars live in the fixed array below, which every GPU that
// loads this library holds until the process exits.

static __device__ __align__(256) unsigned char vx_noalloc_scratch[VX_NOALLOC_SCRATCH_BYTES];

namespace vx {
namespace {

constexpr size_t al256(size_t b) { return (b + 255) & ~size_t(255); }
// r, z, p (two), Ap, then the reduction partials, the scalars, a status word
// and the right-hand side's squared norm
constexpr size_t noalloc_bytes(size_t n) {
    return 5 * al256(3 * n * sizeof(float)) + al256(2 * ((n + kThreads - 1) / kThreads) * sizeof(double)) +
           al256(sizeof(ShimScalars)) + al256(sizeof(uint32_t)) + al256(sizeof(double));
}
static_assert(noalloc_bytes(VX_NOALLOC_MAX_ROWS) <= VX_NOALLOC_SCRATCH_BYTES,
              "the scratch array must hold a system of VX_NOALLOC_MAX_ROWS rows");

// Device address of the scratch array on the current device. Host code cannot
// use the array's name as a device pointer. The address is looked up on every
// call rather than kept: a device reset reloads the module and would leave a
// kept address pointing at memory that no longer exists.
int32_t noalloc_base(char** out) {
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        set_error("vx_solve_pcg_f32_noalloc: no current CUDA device: %s", cudaGetErrorString(e));
        return VX_NO_DEVICE;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, vx_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        set_error("vx_solve_pcg_f32_noalloc: scratch address lookup failed on device %d: %s", device,
                  cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    *out = static_cast<char*>(p);
    return VX_OK;
}

// |rhs|^2 summed by one thread in index order with separate multiply and add
// roundings: the same bits as vx_solve_pcg_f32's host loop, so both entry
// points stop at the same iteration on the same system.
__global__ void k_noalloc_rhs_norm(uint32_t count, const float* __restrict__ rhs, double* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = 0.0;
    for (uint32_t t = 0; t < count; ++t) {
        const double v = (double)rhs[t];
        s = __dadd_rn(s, __dmul_rn(v, v));
    }
    *out = s;
}

// Neighbour slots must name a row of the system (or be empty).
__global__ void k_noalloc_validate(uint32_t n, const uint32_t* __restrict__ nbr6, uint32_t* __restrict__ status) {
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e < 6 * (size_t)n) {
        uint32_t j = nbr6[e];
        if (j != VX_EMPTY_U32 && j >= n) atomicOr(status, 2u);
    }
}

// r = rhs, z = inverse r, dx = 0, p = 0; r.z and r.r.
__global__ void __launch_bounds__(kThreads) k_noalloc_init(ShimArgs a, const float* __restrict__ rhs) {
    uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < a.n) {
        float r[3] = {rhs[3 * (size_t)i], rhs[3 * (size_t)i + 1], rhs[3 * (size_t)i + 2]};
        float z[3];
        m3v(a.inv9 + 9 * (size_t)i, r, z);
        for (int c = 0; c < 3; ++c) {
            a.r[3 * (size_t)i + c] = r[c];
            a.z[3 * (size_t)i + c] = z[c];
            a.dx[3 * (size_t)i + c] = 0.0f;
            const_cast<float*>(a.p_old)[3 * (size_t)i + c] = 0.0f;
        }
        v[0] = dot_ptx(r, z);
        v[1] = dot_ptx(r, r);
    }
    if (grid_sum<2>(v, a.partials, &a.sc->counter[0]) && threadIdx.x == 0) {
        a.sc->rho = v[0];
        a.sc->rr = v[1];
        a.sc->beta = 0.0;
    }
}

__global__ void k_noalloc_finite(uint32_t count, const float* __restrict__ dx, uint32_t* __restrict__ status) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < count && !isfinite(dx[t])) atomicOr(status, 1u);
}

}  // namespace
}  // namespace vx

extern "C" int32_t vx_solve_pcg_f32_noalloc(const float* d_rhs, const uint32_t* d_neighbors,
                                            const float* d_diagonal, const float* d_blocks,
                                            const float* d_inverse_diagonal, uint32_t n, uint32_t max_iterations,
                                            float tolerance, float* d_out_dx, uint32_t* out_iterations,
                                            float* out_relative, void* stream) {
    clear_error();
    if (out_iterations) *out_iterations = 0;
    if (out_relative) *out_relative = 0.0f;
    if (n == 0) return VX_OK;
    if (!d_rhs || !d_neighbors || !d_diagonal || !d_blocks || !d_inverse_diagonal || !d_out_dx) {
        set_error("vx_solve_pcg_f32_noalloc: null argument");
        return VX_BAD_INPUT;
    }
    if (n > VX_NOALLOC_MAX_ROWS) {
        set_error("vx_solve_pcg_f32_noalloc: %u rows exceed the fixed scratch limit of %u rows (%u bytes); "
                  "use vx_solve_pcg_f32 for larger systems",
                  n, (unsigned)VX_NOALLOC_MAX_ROWS, (unsigned)VX_NOALLOC_SCRATCH_BYTES);
        return VX_BAD_INPUT;
    }
    // a non-sticky error left by an earlier, unrelated call on this thread
    // would otherwise be reported as a failure of this call's own launches
    (void)cudaGetLastError();
    char* B = nullptr;
    int32_t st = noalloc_base(&B);
    if (st != VX_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    size_t m = n;
    unsigned blocks_n = (unsigned)((m + kThreads - 1) / kThreads);
    size_t vec = al256(3 * m * sizeof(float));
    size_t off_r = 0, off_z = vec, off_p0 = 2 * vec, off_p1 = 3 * vec, off_ap = 4 * vec, off_part = 5 * vec,
           off_sc = off_part + al256(2 * (size_t)blocks_n * sizeof(double)), off_status = off_sc + al256(sizeof(ShimScalars)),
           off_norm = off_status + al256(sizeof(uint32_t));
    ShimArgs A[2];
    for (int k = 0; k < 2; ++k) {
        A[k].n = n;
        A[k].nbr6 = d_neighbors;
        A[k].diag9 = d_diagonal;
        A[k].blocks54 = d_blocks;
        A[k].inv9 = d_inverse_diagonal;
        A[k].z_in = (const float*)(B + off_z);
        A[k].p_old = (const float*)(B + (k ? off_p1 : off_p0));
        A[k].p_new = (float*)(B + (k ? off_p0 : off_p1));
        A[k].ap = (float*)(B + off_ap);
        A[k].dx = d_out_dx;
        A[k].r = (float*)(B + off_r);
        A[k].z = (float*)(B + off_z);
        A[k].partials = (double*)(B + off_part);
        A[k].sc = (ShimScalars*)(B + off_sc);
    }
    uint32_t* d_status = (uint32_t*)(B + off_status);
    // the array keeps the previous call's contents: the reduction tickets,
    // scalars and status word must start at zero
    cudaError_t e = cudaMemsetAsync(B + off_sc, 0, al256(sizeof(ShimScalars)) + sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        k_noalloc_validate<<<(unsigned)((6 * m + 255) / 256), 256, 0, s>>>(n, d_neighbors, d_status);
        k_noalloc_init<<<blocks_n, kThreads, 0, s>>>(A[0], d_rhs);
        k_noalloc_rhs_norm<<<1, 1, 0, s>>>((uint32_t)(3 * m), d_rhs, (double*)(B + off_norm));
        e = cudaGetLastError();
    }
    ShimScalars h{};
    uint32_t status = 0;
    double initial_sq = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, A[0].sc, sizeof(ShimScalars), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&initial_sq, B + off_norm, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error("vx_solve_pcg_f32_noalloc: set-up failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    if (status & 2u) {
        set_error("vx_solve_pcg_f32_noalloc: a neighbour slot names a row outside the %u-row system", n);
        return VX_BAD_INPUT;
    }
    double initial = std::sqrt(initial_sq);
    if (!(initial > 1e-12)) {
        // (src/cuda_solver.rs:316-324) a zero right-hand side returns a zero correction
        e = cudaMemsetAsync(d_out_dx, 0, 3 * m * sizeof(float), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32_noalloc: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        if (!std::isfinite(initial_sq)) {
            set_error("CUDA PCG produced a non-finite residual norm");
            return VX_NONFINITE;
        }
        return VX_OK;
    }
    uint32_t it = 0;
    double rr = INFINITY;
    int ping = 0;
    while (it < max_iterations) {
        uint32_t step = max_iterations - it < (uint32_t)kShimChunk ? max_iterations - it : (uint32_t)kShimChunk;
        for (uint32_t k = 0; k < step; ++k) {
            k_shim_matvec<<<blocks_n, kThreads, 0, s>>>(A[ping]);
            k_shim_update<<<blocks_n, kThreads, 0, s>>>(A[ping]);
            ping ^= 1;
        }
        it += step;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, A[0].sc, sizeof(ShimScalars), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error("vx_solve_pcg_f32_noalloc: iteration failed: %s", cudaGetErrorString(e));
            return VX_CUDA_ERROR;
        }
        rr = h.rr;
        if (!std::isfinite(rr) || rr < 0.0) break;
        if ((float)(std::sqrt(rr) / initial) <= tolerance) break;
    }
    if (out_iterations) *out_iterations = it;
    if (!std::isfinite(rr) || rr < 0.0) {
        set_error("CUDA PCG produced a non-finite residual norm");
        return VX_NONFINITE;
    }
    float relative = (float)(std::sqrt(rr) / initial);
    if (out_relative) *out_relative = relative;
    if (!std::isfinite(relative) || relative > tolerance) {
        set_error("CUDA PCG did not converge: iterations=%u, relative residual=%.3e, tolerance=%.3e", it, relative,
                  tolerance);
        return VX_NOT_CONVERGED;
    }
    k_noalloc_finite<<<(unsigned)((3 * m + 255) / 256), 256, 0, s>>>((uint32_t)(3 * m), d_out_dx, d_status);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error("vx_solve_pcg_f32_noalloc: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    if (status & 1u) {
        set_error("CUDA PCG produced a non-finite correction");
        return VX_NONFINITE;
    }
    return VX_OK;
}
