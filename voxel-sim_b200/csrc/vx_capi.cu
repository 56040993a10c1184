// vx_capi.cu — extern "C" entry points of include/vxcorot.h (scene API).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vx_kernels.h"
#include "vx_layout.cuh"

namespace vx {

static thread_local std::string g_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}
void clear_error() { g_error.clear(); }

void scene_release(vx_scene* s);

// Carves every device array of a scene out of one allocation. With a null
// base it only measures.
static void carve(vx_scene* s, Arena& A, uint32_t n, uint32_t mc) {
    size_t m = n ? n : 1;
    unsigned blocks = (unsigned)((m + 255) / 256);
    s->pos = A.take<double>(3 * m);
    s->pred = A.take<double>(3 * m);
    s->loads = A.take<double>(3 * m);
    s->target = A.take<double>(3 * m);
    s->rot = A.take<double4>(m);
    s->kin = A.take<uint8_t>(m);
    s->tmask = A.take<uint8_t>(m);
    s->flags = A.take<uint8_t>(m);
    s->param0 = A.take<float4>(m);
    s->param1 = A.take<float4>(m);
    s->matid = A.take<uint32_t>(m);
    s->materials = A.take<vx_material>(mc ? mc : 1);
    s->nbr = A.take<uint32_t>(3 * m);
    s->rev = A.take<uint32_t>(3 * m);
    s->bond_a = A.take<float4>(3 * m);
    s->bond_b = A.take<float4>(3 * m);
    s->bond_c = A.take<float4>(3 * m);
    s->bond_d = A.take<float>(3 * m);
    s->last_force = A.take<float>(9 * m);
    s->frac_partials = A.take<double>(5 * 3 * (size_t)blocks);
    s->frac_totals = A.take<double>(8);
    s->frac_counter = A.take<uint32_t>(2);
    s->clusters = A.take<uint32_t>(m);
    s->cl_parent = A.take<uint32_t>(m);
    s->cl_root = A.take<uint32_t>(m);
    s->cl_first = A.take<uint32_t>(m);
    s->cl_scan = A.take<uint32_t>(m);
    s->cl_bsum = A.take<uint32_t>(m / 1024 + 2);
    s->cl_err = A.take<uint32_t>(1);
    s->bonds.k64 = A.take<double>(18 * m);
    s->bonds.k32 = A.take<float>(18 * (size_t)kstride32((uint32_t)m));
    s->bonds.mat_k = A.take<double>(18 * m);
    s->bonds.frame_q = A.take<double4>(3 * m);
    s->bonds.force = A.take<double>(9 * m);
    s->bonds.state = A.take<uint8_t>(3 * m);
    s->d64 = A.take<double>(6 * m);
    s->dinv64 = A.take<double>(6 * m);
    s->d32 = A.take<float>(6 * m);
    s->mh2_32 = A.take<float>(m);
    s->dinv32 = A.take<float>(6 * m);
    s->b64 = A.take<double>(3 * m);
    s->x64 = A.take<double>(3 * m);
    s->r64 = A.take<double>(3 * m);
    s->z64 = A.take<double>(3 * m);
    s->p64[0] = A.take<double>(3 * m);
    s->p64[1] = A.take<double>(3 * m);
    s->ap64 = A.take<double>(3 * m);
    s->x32 = A.take<float>(3 * m);
    s->r32 = A.take<float>(3 * m);
    s->z32 = A.take<float>(3 * m);
    s->p32[0] = A.take<float>(3 * m);
    s->p32[1] = A.take<float>(3 * m);
    s->ap32 = A.take<float>(3 * m);
    s->vel = A.take<double>(3 * m);
    s->prev = A.take<double>(3 * m);
    s->drift = A.take<double>(3 * m);
    s->rest = A.take<float>(3 * m);
    s->save_pos = A.take<double>(3 * m);
    s->save_rot = A.take<double4>(m);
    s->out_ratio = A.take<float>(3 * m);
    s->out_force = A.take<float>(9 * m);
    s->out_near = A.take<uint32_t>(3 * m);
    s->partials = A.take<double>(4 * (size_t)blocks);
    s->sc = A.take<PcgScalars>(1);
    s->sc32 = A.take<PcgScalars>(1);
    s->max_angle_bits = A.take<unsigned long long>(1);
    s->near_count = A.take<uint32_t>(1);
    s->bond_count = A.take<uint32_t>(1);
    s->barrier = A.take<unsigned>(4);
    s->zp32 = A.take<float>(6 * m);
    s->nbcode = A.take<uint32_t>(3 * m);
    s->nbcode_bad = A.take<uint32_t>(2);  // [0] neighbour deltas out of range, [1] upload check
}

uint64_t scene_bytes(uint32_t n, uint32_t material_count) {
    vx_scene probe;
    Arena A;
    carve(&probe, A, n, material_count);
    return A.used;
}

static int32_t cuda_fail(cudaError_t e, const char* what) {
    set_error("%s failed: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return VX_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return VX_NO_DEVICE;
    return VX_CUDA_ERROR;
}

#define VX_TRY(expr, what)                              \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

// AoS (n x 3) <-> SoA [3][n] on the device: the host only makes contiguous
// copies, and one kernel reorders.
__global__ void k_aos_to_soa(size_t n, const double* __restrict__ aos, double* __restrict__ soa) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;  // t = 3 i + c, coalesced reads
    if (t < 3 * n) soa[(t % 3) * n + t / 3] = aos[t];
}
__global__ void k_soa_to_aos(size_t n, const double* __restrict__ soa, double* __restrict__ aos) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;  // t = 3 i + c, coalesced writes
    if (t < 3 * n) aos[t] = soa[(t % 3) * n + t / 3];
}
// Counts the non-finite values of v[count] into *bad.
__global__ void k_count_nonfinite(size_t count, const double* __restrict__ v, uint32_t* bad) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const bool nf = t < count && !isfinite(v[t]);
    const unsigned ballot = __ballot_sync(0xffffffffu, nf);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(bad, (uint32_t)__popc(ballot));
}

// Page-locked host memory (cudaMallocHost or registered) is copied by DMA
// directly; other host memory goes through the scene's pinned stage.
static bool is_pinned(const void* p) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}
// Host bytes -> device (through the stage unless the source is pinned).
static cudaError_t host_to_device(vx_scene* s, void* dst, const void* src, size_t bytes) {
    if (is_pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream);
    cudaError_t e = cudaStreamSynchronize(s->stream);  // the stage may still feed a copy
    if (e != cudaSuccess) return e;
    std::memcpy(s->h_stage, src, bytes);
    return cudaMemcpyAsync(dst, s->h_stage, bytes, cudaMemcpyHostToDevice, s->stream);
}
// Device bytes -> host; returns after the copy has landed.
static cudaError_t device_to_host(vx_scene* s, void* dst, const void* src, size_t bytes) {
    if (is_pinned(dst)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream);
        return e == cudaSuccess ? cudaStreamSynchronize(s->stream) : e;
    }
    cudaError_t e = cudaMemcpyAsync(s->h_stage, src, bytes, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) std::memcpy(dst, s->h_stage, bytes);
    return e;
}

// AoS host doubles -> SoA device doubles. The transit buffer is the FP64
// residual vector r64, which holds nothing between solves (every host call on
// a scene runs on its stream, between solves). With check_finite, nothing is
// written and VX_NONFINITE is returned when a value is not finite.
static int32_t upload_vec3(vx_scene* s, double* dst, const double* src, bool check_finite = false,
                           const char* what = "upload") {
    const size_t n = s->n, bytes = 3 * n * sizeof(double);
    if (n == 0) return VX_OK;
    VX_TRY(host_to_device(s, s->r64, src, bytes), what);
    if (check_finite) {
        VX_TRY(cudaMemsetAsync(s->nbcode_bad + 1, 0, sizeof(uint32_t), s->stream), what);
        k_count_nonfinite<<<(unsigned)((3 * n + 255) / 256), 256, 0, s->stream>>>(3 * n, s->r64, s->nbcode_bad + 1);
        uint32_t bad = 0;
        VX_TRY(device_to_host(s, &bad, s->nbcode_bad + 1, sizeof(uint32_t)), what);
        if (bad) {
            set_error("%s: %u non-finite values", what, bad);
            return VX_NONFINITE;
        }
    }
    k_aos_to_soa<<<(unsigned)((3 * n + 255) / 256), 256, 0, s->stream>>>(n, s->r64, dst);
    VX_TRY(cudaGetLastError(), "upload reorder");
    VX_TRY(cudaStreamSynchronize(s->stream), "upload sync");
    return VX_OK;
}
static int32_t download_vec3(vx_scene* s, double* dst, const double* src) {
    const size_t n = s->n, bytes = 3 * n * sizeof(double);
    if (n == 0) return VX_OK;
    k_soa_to_aos<<<(unsigned)((3 * n + 255) / 256), 256, 0, s->stream>>>(n, src, s->r64);
    VX_TRY(cudaGetLastError(), "download reorder");
    VX_TRY(device_to_host(s, dst, s->r64, bytes), "download");
    return VX_OK;
}

// Allocates a scene's arena (n REVs, material_count materials), its stream and
// pinned host buffers (a stage of 4 doubles per REV, for at most stage_revs
// REVs when that is not 0), and clears the arena.
int32_t scene_alloc(vx_scene* s, vx_ctx* ctx, uint32_t n, uint32_t material_count, size_t stage_revs) {
    s->ctx = ctx;
    s->device = ctx->device;
    s->sm_count = ctx->sm_count > 0 ? ctx->sm_count : 1;
    s->n = n;
    s->blocks = (n + 255) / 256;
    s->material_count = material_count;
    Arena probe;
    carve(s, probe, n, material_count);
    cudaError_t e = cudaMalloc(&s->arena.base, probe.used);
    if (e != cudaSuccess) return cuda_fail(e, "scene allocation");
    s->arena.size = probe.used;
    s->arena.used = 0;
    carve(s, s->arena, n, material_count);
    e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    size_t stage = n ? n : 1;
    if (stage_revs && stage_revs < stage) stage = stage_revs;
    s->stage_revs = stage;
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_stage, 4 * stage * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_sc, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_done, 2 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev[1], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->arena.base, 0, s->arena.size, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        int32_t st = cuda_fail(e, "scene set-up");
        scene_release(s);
        return st;
    }
    return VX_OK;
}

void scene_release(vx_scene* s) {
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    contact_release(s);
    if (s->chunk64) cudaGraphExecDestroy(s->chunk64);
    if (s->chunk32) cudaGraphExecDestroy(s->chunk32);
    for (int k = 0; k < 2; ++k)
        if (s->ev[k]) cudaEventDestroy(s->ev[k]);
    if (s->h_sc) cudaFreeHost(s->h_sc);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_stage) cudaFreeHost(s->h_stage);
    if (s->arena.base) cudaFree(s->arena.base);
    if (s->brick_buf) cudaFree(s->brick_buf);
    s->brick_buf = nullptr;
    if (s->exp_buf) cudaFree(s->exp_buf);
    s->exp_buf = nullptr;
    s->brick_ok = false;
    if (s->stream) cudaStreamDestroy(s->stream);
    s->chunk64 = s->chunk32 = nullptr;
    s->ev[0] = s->ev[1] = nullptr;
    s->h_sc = nullptr;
    s->h_done = nullptr;
    s->h_stage = nullptr;
    s->arena.base = nullptr;
    s->stream = nullptr;
}

// Shared by the single-scene and pool steps: one fracture stage, then the
// reverse table and neighbour deltas when a bond broke.
int32_t fracture_stage(vx_scene* s, double dt, const vx_fracture_config* cfg, vx_dissipation* out,
                       uint32_t* out_broken) {
    if (!s->assembled) {
        set_error("vx_fracture_commit: no corotational pass has assembled the bonds yet");
        return VX_BAD_INPUT;
    }
    VX_TRY(launch_fracture_commit(s, dt, cfg), "fracture launch");
    double tot[8];
    uint32_t cnt[2];
    VX_TRY(cudaMemcpyAsync(tot, s->frac_totals, sizeof tot, cudaMemcpyDeviceToHost, s->stream), "fracture");
    VX_TRY(cudaMemcpyAsync(cnt, s->frac_counter, sizeof cnt, cudaMemcpyDeviceToHost, s->stream), "fracture");
    VX_TRY(cudaStreamSynchronize(s->stream), "fracture");
    if (cnt[1]) {
        VX_TRY(launch_reverse_neighbors(s), "reverse neighbours");
        VX_TRY(cudaStreamSynchronize(s->stream), "reverse neighbours");
    }
    if (out) *out = vx_dissipation{tot[0], tot[1], tot[2], tot[3], tot[4]};
    if (out_broken) *out_broken = cnt[1];
    return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" {

const char* vx_last_error(void) { return g_error.c_str(); }
int32_t vx_abi_version(void) { return VX_ABI_VERSION; }

int32_t vx_ctx_create(int32_t device, vx_ctx** out_ctx) {
    clear_error();
    if (!out_ctx) {
        set_error("vx_ctx_create: null output");
        return VX_BAD_INPUT;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_error("vx_ctx_create: no CUDA device (%s)", cudaGetErrorString(e));
        return VX_NO_DEVICE;
    }
    if (device < 0 || device >= count) {
        set_error("vx_ctx_create: device %d out of range (%d devices)", device, count);
        return VX_BAD_INPUT;
    }
    VX_TRY(cudaSetDevice(device), "cudaSetDevice");
    vx_ctx* c = new (std::nothrow) vx_ctx();
    if (!c) return VX_OOM;
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate");
    }
    *out_ctx = c;
    return VX_OK;
}

int32_t vx_ctx_destroy(vx_ctx* ctx) {
    if (!ctx) return VX_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return VX_OK;
}

uint64_t vx_scene_footprint_bytes(uint32_t n) { return scene_bytes(n, 16); }

int32_t vx_build_topology(vx_ctx* ctx, const int32_t* cells, const uint8_t* kinematic, uint32_t n,
                          uint32_t* out_neighbor) {
    clear_error();
    if (!ctx || (n && (!cells || !kinematic || !out_neighbor))) {
        set_error("vx_build_topology: null argument");
        return VX_BAD_INPUT;
    }
    if (n == 0) return VX_OK;
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = cells[a];
    for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], cells[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], cells[3 * (size_t)i + a]);
        }
    int32_t ext[3];
    double vol = 1.0;
    for (int a = 0; a < 3; ++a) {
        ext[a] = hi[a] - lo[a] + 2;  // one spare layer on the + side
        vol *= ext[a];
    }
    if (vol > 2.0e9) {
        set_error("vx_build_topology: lattice bounding box of %.3g cells is too large", vol);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(ctx->device);
    size_t cells_b = 3 * (size_t)n * sizeof(int32_t), grid_b = (size_t)vol * sizeof(int32_t);
    char* buf = nullptr;
    size_t total = cells_b + n + grid_b + 3 * (size_t)n * sizeof(uint32_t) + 256 * 4;
    VX_TRY(cudaMalloc(&buf, total), "topology allocation");
    int32_t* d_cells = (int32_t*)buf;
    int32_t* d_grid = (int32_t*)(buf + ((cells_b + 255) & ~size_t(255)));
    uint32_t* d_nbr = (uint32_t*)((char*)d_grid + ((grid_b + 255) & ~size_t(255)));
    uint8_t* d_kin = (uint8_t*)((char*)d_nbr + ((3 * (size_t)n * 4 + 255) & ~size_t(255)));
    uint32_t* d_dup = (uint32_t*)(d_kin + ((n + 255) & ~size_t(255)));
    if ((char*)(d_dup + 1) > buf + total) {
        cudaFree(buf);
        set_error("vx_build_topology: internal layout error");
        return VX_CUDA_ERROR;
    }
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_cells, cells, cells_b, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_kin, kinematic, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_grid, 0xFF, grid_b, st);
    if (e == cudaSuccess) e = launch_topology(d_cells, d_kin, n, lo, ext, d_grid, d_nbr, d_dup, st);
    uint32_t dup = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_neighbor, d_nbr, 3 * (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&dup, d_dup, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "vx_build_topology");
    if (dup) {
        set_error("vx_build_topology: %u duplicate lattice cells", dup);
        return VX_BAD_INPUT;
    }
    return VX_OK;
}

int32_t vx_scene_create(vx_ctx* ctx, const vx_scene_desc* d, vx_scene** out) {
    clear_error();
    if (!ctx || !d || !out) {
        set_error("vx_scene_create: null argument");
        return VX_BAD_INPUT;
    }
    uint32_t n = d->n;
    if (n && (!d->position || !d->kinematic || !d->mass || !d->material || !d->materials || !d->fiber ||
              !d->anisotropy || !d->neighbor)) {
        set_error("vx_scene_create: a required array is null");
        return VX_BAD_INPUT;
    }
    if (n >= 0x7FFFFFFFu / 3) {
        set_error("vx_scene_create: %u REVs exceed the index range", n);
        return VX_BAD_INPUT;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (d->material[i] >= d->material_count) {
            set_error("vx_scene_create: REV %u has material %u of %u", i, d->material[i], d->material_count);
            return VX_BAD_INPUT;
        }
        for (int c = 0; c < 3; ++c) {
            if (!std::isfinite(d->position[3 * (size_t)i + c])) {
                set_error("vx_scene_create: non-finite position of REV %u", i);
                return VX_NONFINITE;
            }
        }
    }
    for (size_t e = 0; e < 3 * (size_t)n; ++e) {
        uint32_t j = d->neighbor[e];
        if (j != VX_EMPTY && j >= n) {
            set_error("vx_scene_create: bond %zu points at REV %u of %u", e, j, n);
            return VX_BAD_INPUT;
        }
    }
    cudaSetDevice(ctx->device);
    vx_scene* s = new (std::nothrow) vx_scene();
    if (!s) return VX_OOM;
    int32_t ar = scene_alloc(s, ctx, n, d->material_count, 0);
    if (ar != VX_OK) {
        delete s;
        return ar;
    }
    auto fail = [&](cudaError_t err, const char* what) {
        int32_t st = cuda_fail(err, what);
        vx_scene_destroy(s);
        return st;
    };
    cudaError_t e = cudaSuccess;
    size_t m = n;
    // host staging in device layout
    std::vector<double4> rot(m);
    std::vector<float4> p0(m), p1(m), ba(3 * m), bb(3 * m);
    for (size_t i = 0; i < m; ++i) {
        if (d->rotation)
            rot[i] = make_double4(d->rotation[4 * i], d->rotation[4 * i + 1], d->rotation[4 * i + 2],
                                  d->rotation[4 * i + 3]);
        else
            rot[i] = make_double4(0.0, 0.0, 0.0, 1.0);
        p0[i] = make_float4(d->fiber[3 * i], d->fiber[3 * i + 1], d->fiber[3 * i + 2], d->anisotropy[i]);
        p1[i] = make_float4(d->solid_fraction ? d->solid_fraction[i] : 1.0f,
                            d->thermal_strength ? d->thermal_strength[i] : 1.0f,
                            d->thermal_delta ? d->thermal_delta[i] : 0.0f, d->mass[i]);
    }
    for (size_t e2 = 0; e2 < 3 * m; ++e2) {
        float fo[3] = {0, 0, 0}, pl[3] = {0, 0, 0};
        if (d->formation_offset)
            for (int c = 0; c < 3; ++c) fo[c] = d->formation_offset[3 * e2 + c];
        if (d->plastic_strain)
            for (int c = 0; c < 3; ++c) pl[c] = d->plastic_strain[3 * e2 + c];
        ba[e2] = make_float4(fo[0], fo[1], fo[2], d->damage ? d->damage[e2] : 0.0f);
        bb[e2] = make_float4(pl[0], pl[1], pl[2], 0.0f);
    }
    cudaStream_t st = s->stream;
    if (n) {
        e = cudaMemcpyAsync(s->rot, rot.data(), m * sizeof(double4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->param0, p0.data(), m * sizeof(float4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->param1, p1.data(), m * sizeof(float4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->bond_a, ba.data(), 3 * m * sizeof(float4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->bond_b, bb.data(), 3 * m * sizeof(float4), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->kin, d->kinematic, m, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->matid, d->material, m * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->nbr, d->neighbor, 3 * m * 4, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(e, "scene upload");
    }
    if (d->material_count) {
        e = cudaMemcpyAsync(s->materials, d->materials, d->material_count * sizeof(vx_material),
                            cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(e, "material upload");
    }
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "scene upload");
    if (n) {
        int32_t r = upload_vec3(s, s->pos, d->position);
        if (r != VX_OK) {
            vx_scene_destroy(s);
            return r;
        }
        e = cudaMemcpyAsync(s->pred, s->pos, 3 * m * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->prev, s->pos, 3 * m * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = launch_rest_positions(s);
        if (e == cudaSuccess) e = launch_reverse_neighbors(s);
        if (e == cudaSuccess) e = launch_flags(s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(e, "scene setup");
    }
    *out = s;
    return VX_OK;
}

int32_t vx_scene_destroy(vx_scene* s) {
    if (!s) return VX_OK;
    scene_release(s);
    delete s;
    return VX_OK;
}

#define VX_CHECK_SCENE(s, p)                                      \
    do {                                                          \
        clear_error();                                            \
        if (!(s) || (!(p) && (s)->n)) {                           \
            set_error("%s: null argument", __func__);             \
            return VX_BAD_INPUT;                                  \
        }                                                         \
        cudaSetDevice((s)->device);                          \
    } while (0)

int32_t vx_scene_set_positions(vx_scene* s, const double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return upload_vec3(s, s->pos, xyz, true, "vx_scene_set_positions");
}
int32_t vx_scene_set_previous(vx_scene* s, const double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return upload_vec3(s, s->prev, xyz, true, "vx_scene_set_previous");
}
int32_t vx_scene_get_positions(vx_scene* s, double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return download_vec3(s, xyz, s->pos);
}
int32_t vx_scene_set_rotations(vx_scene* s, const double* q) {
    VX_CHECK_SCENE(s, q);
    if (s->n == 0) return VX_OK;
    VX_TRY(host_to_device(s, s->rot, q, (size_t)s->n * sizeof(double4)), "upload");
    VX_TRY(cudaStreamSynchronize(s->stream), "upload");
    return VX_OK;
}
int32_t vx_scene_get_rotations(vx_scene* s, double* q) {
    VX_CHECK_SCENE(s, q);
    if (s->n == 0) return VX_OK;
    VX_TRY(device_to_host(s, q, s->rot, (size_t)s->n * sizeof(double4)), "download");
    return VX_OK;
}
int32_t vx_scene_set_targets(vx_scene* s, const uint8_t* mask, const double* xyz) {
    VX_CHECK_SCENE(s, mask);
    VX_TRY(cudaMemcpyAsync(s->tmask, mask, s->n, cudaMemcpyHostToDevice, s->stream), "upload");
    if (xyz) {
        int32_t r = upload_vec3(s, s->target, xyz);
        if (r != VX_OK) return r;
    }
    VX_TRY(launch_flags(s), "flags");
    VX_TRY(cudaStreamSynchronize(s->stream), "upload");
    s->active_cached = false;
    return VX_OK;
}
int32_t vx_scene_set_velocities(vx_scene* s, const double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return upload_vec3(s, s->vel, xyz, true, "vx_scene_set_velocities");
}
int32_t vx_scene_get_velocities(vx_scene* s, double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return download_vec3(s, xyz, s->vel);
}
int32_t vx_scene_update_velocities(vx_scene* s, uint32_t count, const uint32_t* index, const double* value,
                                   int32_t op) {
    clear_error();
    if (!s || (count && (!index || !value)) || (op != 0 && op != 1)) {
        set_error("vx_scene_update_velocities: bad argument");
        return VX_BAD_INPUT;
    }
    for (uint32_t k = 0; k < count; ++k) {
        if (index[k] >= s->n) {
            set_error("vx_scene_update_velocities: index %u out of range", index[k]);
            return VX_BAD_INPUT;
        }
        for (int a = 0; a < 3; ++a)
            if (!std::isfinite(value[3 * (size_t)k + a])) {
                set_error("vx_scene_update_velocities: non-finite value for REV %u", index[k]);
                return VX_NONFINITE;
            }
    }
    if (count == 0) return VX_OK;
    cudaSetDevice(s->device);
    // values and indices travel through the pinned stage (3 + 1 doubles per
    // entry, at most n entries at a time) into the FP64 z and p vectors, which
    // are free between passes
    for (uint32_t base = 0; base < count;) {
        const uint32_t chunk = (uint32_t)std::min<size_t>(count - base, s->stage_revs);
        VX_TRY(cudaStreamSynchronize(s->stream), "velocity update");
        double* vals = s->h_stage;
        uint32_t* idx = reinterpret_cast<uint32_t*>(s->h_stage + 3 * (size_t)chunk);
        std::memcpy(vals, value + 3 * (size_t)base, 3 * (size_t)chunk * sizeof(double));
        std::memcpy(idx, index + base, (size_t)chunk * sizeof(uint32_t));
        double* d_vals = s->z64;
        uint32_t* d_idx = reinterpret_cast<uint32_t*>(s->p64[0]);
        VX_TRY(cudaMemcpyAsync(d_vals, vals, 3 * (size_t)chunk * sizeof(double), cudaMemcpyHostToDevice, s->stream),
               "velocity update");
        VX_TRY(cudaMemcpyAsync(d_idx, idx, (size_t)chunk * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream),
               "velocity update");
        VX_TRY(launch_velocity_update(s, chunk, d_idx, d_vals, op), "velocity update");
        base += chunk;
    }
    VX_TRY(cudaStreamSynchronize(s->stream), "velocity update");
    return VX_OK;
}
// Indexed reads and writes of a per-REV vector field, staged in chunks of at
// most n entries through the pinned stage and the FP64 z / p solver vectors
// (free between passes).
static int32_t indexed_field(vx_scene* s, int32_t field, uint32_t count, const uint32_t* index, double* xyz,
                             bool write, const char* who) {
    clear_error();
    if (!s || (count && (!index || !xyz)) || (field != VX_FIELD_POSITION && field != VX_FIELD_VELOCITY && field != VX_FIELD_PREVIOUS)) {
        set_error("%s: bad argument", who);
        return VX_BAD_INPUT;
    }
    for (uint32_t k = 0; k < count; ++k) {
        if (index[k] >= s->n) {
            set_error("%s: index %u out of range", who, index[k]);
            return VX_BAD_INPUT;
        }
        if (write)
            for (int a = 0; a < 3; ++a)
                if (!std::isfinite(xyz[3 * (size_t)k + a])) {
                    set_error("%s: non-finite value for REV %u", who, index[k]);
                    return VX_NONFINITE;
                }
    }
    if (count == 0) return VX_OK;
    cudaSetDevice(s->device);
    double* dev_field = field == VX_FIELD_POSITION ? s->pos : (field == VX_FIELD_VELOCITY ? s->vel : s->prev);
    for (uint32_t base = 0; base < count;) {
        const uint32_t chunk = (uint32_t)std::min<size_t>(count - base, s->stage_revs);
        VX_TRY(cudaStreamSynchronize(s->stream), who);
        double* vals = s->h_stage;
        uint32_t* idx = reinterpret_cast<uint32_t*>(s->h_stage + 3 * (size_t)chunk);
        std::memcpy(idx, index + base, (size_t)chunk * sizeof(uint32_t));
        double* d_vals = s->z64;
        uint32_t* d_idx = reinterpret_cast<uint32_t*>(s->p64[0]);
        VX_TRY(cudaMemcpyAsync(d_idx, idx, (size_t)chunk * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream), who);
        if (write) {
            std::memcpy(vals, xyz + 3 * (size_t)base, 3 * (size_t)chunk * sizeof(double));
            VX_TRY(cudaMemcpyAsync(d_vals, vals, 3 * (size_t)chunk * sizeof(double), cudaMemcpyHostToDevice,
                                   s->stream), who);
            VX_TRY(launch_scatter3(s, chunk, d_idx, d_vals, dev_field), who);
        } else {
            VX_TRY(launch_gather3(s, chunk, d_idx, dev_field, d_vals), who);
            VX_TRY(cudaMemcpyAsync(vals, d_vals, 3 * (size_t)chunk * sizeof(double), cudaMemcpyDeviceToHost,
                                   s->stream), who);
            VX_TRY(cudaStreamSynchronize(s->stream), who);
            std::memcpy(xyz + 3 * (size_t)base, vals, 3 * (size_t)chunk * sizeof(double));
        }
        base += chunk;
    }
    VX_TRY(cudaStreamSynchronize(s->stream), who);
    return VX_OK;
}
int32_t vx_scene_read_revs(vx_scene* s, int32_t field, uint32_t count, const uint32_t* index, double* xyz) {
    return indexed_field(s, field, count, index, xyz, false, "vx_scene_read_revs");
}
int32_t vx_scene_write_revs(vx_scene* s, int32_t field, uint32_t count, const uint32_t* index, const double* xyz) {
    return indexed_field(s, field, count, index, const_cast<double*>(xyz), true, "vx_scene_write_revs");
}
int32_t vx_scene_set_loads(vx_scene* s, const double* xyz) {
    VX_CHECK_SCENE(s, xyz);
    return upload_vec3(s, s->loads, xyz);
}
int32_t vx_scene_set_predicted(vx_scene* s, const double* xyz) {
    clear_error();
    if (!s) return VX_BAD_INPUT;
    cudaSetDevice(s->device);
    if (!xyz) {
        VX_TRY(cudaMemcpyAsync(s->pred, s->pos, 3 * (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice,
                               s->stream), "predicted");
        VX_TRY(cudaStreamSynchronize(s->stream), "predicted");
        return VX_OK;
    }
    return upload_vec3(s, s->pred, xyz);
}
int32_t vx_scene_set_bonds(vx_scene* s, const uint32_t* neighbor, const float* plastic, const float* damage,
                           const float* formation) {
    VX_CHECK_SCENE(s, neighbor);
    size_t m = 3 * (size_t)s->n;
    for (size_t e = 0; e < m; ++e)
        if (neighbor[e] != VX_EMPTY && neighbor[e] >= s->n) {
            set_error("vx_scene_set_bonds: bond %zu points at REV %u of %u", e, neighbor[e], s->n);
            return VX_BAD_INPUT;
        }
    std::vector<float4> ba(m), bb(m);
    for (size_t e = 0; e < m; ++e) {
        ba[e] = make_float4(formation ? formation[3 * e] : 0.f, formation ? formation[3 * e + 1] : 0.f,
                            formation ? formation[3 * e + 2] : 0.f, damage ? damage[e] : 0.f);
        bb[e] = make_float4(plastic ? plastic[3 * e] : 0.f, plastic ? plastic[3 * e + 1] : 0.f,
                            plastic ? plastic[3 * e + 2] : 0.f, 0.f);
    }
    VX_TRY(cudaMemcpyAsync(s->nbr, neighbor, m * 4, cudaMemcpyHostToDevice, s->stream), "upload");
    VX_TRY(cudaMemcpyAsync(s->bond_a, ba.data(), m * sizeof(float4), cudaMemcpyHostToDevice, s->stream), "upload");
    VX_TRY(cudaMemcpyAsync(s->bond_b, bb.data(), m * sizeof(float4), cudaMemcpyHostToDevice, s->stream), "upload");
    VX_TRY(launch_reverse_neighbors(s), "reverse neighbours");
    VX_TRY(cudaStreamSynchronize(s->stream), "upload");
    return VX_OK;
}
int32_t vx_scene_get_neighbors(vx_scene* s, uint32_t* neighbor) {
    VX_CHECK_SCENE(s, neighbor);
    VX_TRY(cudaMemcpyAsync(neighbor, s->nbr, 3 * (size_t)s->n * 4, cudaMemcpyDeviceToHost, s->stream), "download");
    VX_TRY(cudaStreamSynchronize(s->stream), "download");
    return VX_OK;
}

int32_t vx_fit_rotations(vx_scene* s, double* out_max_angle) {
    clear_error();
    if (!s) return VX_BAD_INPUT;
    cudaSetDevice(s->device);
    VX_TRY(launch_fit_rotations(s), "fit_rotations launch");
    unsigned long long bits = 0;
    VX_TRY(cudaMemcpyAsync(&bits, s->max_angle_bits, 8, cudaMemcpyDeviceToHost, s->stream), "fit_rotations");
    VX_TRY(cudaStreamSynchronize(s->stream), "fit_rotations");
    double v;
    std::memcpy(&v, &bits, 8);
    if (out_max_angle) *out_max_angle = v;
    return VX_OK;
}

static uint32_t count_active(vx_scene* s) {
    if (s->active_cached) return s->active;
    std::vector<uint8_t> fl(s->n);
    if (s->n) {
        cudaMemcpy(fl.data(), s->flags, s->n, cudaMemcpyDeviceToHost);
    }
    uint32_t a = 0;
    for (uint8_t f : fl) a += f != 0;
    s->active = a;
    s->active_cached = true;
    return a;
}

int32_t vx_corotational_pass(vx_scene* s, const vx_pass_params* p, vx_pass_stats* out) {
    clear_error();
    if (!s || !p) {
        set_error("vx_corotational_pass: null argument");
        return VX_BAD_INPUT;
    }
    if (!(p->h > 0.0) || !std::isfinite(p->h) || !(p->tolerance > 0.0)) {
        set_error("vx_corotational_pass: invalid h=%g or tolerance=%g", p->h, p->tolerance);
        return VX_BAD_INPUT;
    }
    if (p->kernel < VX_KERNEL_AUTO || p->kernel > VX_KERNEL_PERSISTENT) {
        set_error("vx_corotational_pass: unknown kernel selection %d", p->kernel);
        return VX_BAD_INPUT;
    }
    if (p->precision != VX_PRECISION_FP64 && p->precision != VX_PRECISION_MIXED) {
        set_error("vx_corotational_pass: unknown precision %d", p->precision);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    vx_pass_stats st{};
    bool reuse = p->reuse_preconditioner && s->have_dinv;
    s->launches = 2;
    VX_TRY(launch_assembly(s, p->h, reuse), "assembly launch");
    s->have_dinv = true;
    s->assembled = true;
    int32_t status;
    if (p->precision == VX_PRECISION_FP64)
        status = solve_fp64(s, p->tolerance, p->max_iterations, &st);
    else
        status = solve_mixed(s, p->tolerance, p->max_iterations, p->inner_tolerance, p->max_outer, p->kernel, &st);
    if (status == VX_CUDA_ERROR) return status;
    double tr = 0.0;
    int32_t r = true_residual(s, &tr);
    if (r != VX_OK) return r;
    st.true_residual = tr;
    if (p->precision == VX_PRECISION_MIXED) st.residual = tr;
    VX_TRY(launch_apply_correction(s), "correction");
    VX_TRY(cudaStreamSynchronize(s->stream), "pass");
    st.kernel_launches = s->launches + 2;
    st.active = count_active(s);
    VX_TRY(cudaMemcpy(&st.bonds_assembled, s->bond_count, 4, cudaMemcpyDeviceToHost), "pass stats");
    if (out) *out = st;
    if (status == VX_NONFINITE) set_error("vx_corotational_pass: non-finite value in the solve");
    else if (status == VX_NOT_CONVERGED)
        set_error("vx_corotational_pass: not converged after %u iterations, residual %.3e", st.iterations,
                  st.residual);
    return status;
}

int32_t vx_bond_stress(vx_scene* s, float* ratio, float* force, uint32_t* near, uint32_t cap,
                       uint32_t* near_count) {
    clear_error();
    if (!s) return VX_BAD_INPUT;
    if (!s->assembled) {
        set_error("vx_bond_stress: no corotational pass has assembled the bonds yet");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    size_t m = 3 * (size_t)s->n;
    VX_TRY(launch_bond_stress(s, s->out_ratio, force ? s->out_force : nullptr, s->out_near, (uint32_t)m),
           "bond stress launch");
    uint32_t count = 0;
    VX_TRY(cudaMemcpyAsync(&count, s->near_count, 4, cudaMemcpyDeviceToHost, s->stream), "bond stress");
    if (ratio) VX_TRY(cudaMemcpyAsync(ratio, s->out_ratio, m * 4, cudaMemcpyDeviceToHost, s->stream), "bond stress");
    if (force)
        VX_TRY(cudaMemcpyAsync(force, s->out_force, 3 * m * 4, cudaMemcpyDeviceToHost, s->stream), "bond stress");
    VX_TRY(cudaStreamSynchronize(s->stream), "bond stress");
    if (near && cap) {
        std::vector<uint32_t> tmp(std::min<uint32_t>(count, (uint32_t)m));
        if (!tmp.empty()) {
            VX_TRY(cudaMemcpy(tmp.data(), s->out_near, tmp.size() * 4, cudaMemcpyDeviceToHost), "near list");
            std::sort(tmp.begin(), tmp.end());
        }
        for (size_t k = 0; k < tmp.size() && k < cap; ++k) near[k] = tmp[k];
    }
    if (near_count) *near_count = count;
    return VX_OK;
}

int32_t vx_fracture_commit(vx_scene* s, double dt, const vx_fracture_config* cfg, vx_dissipation* out,
                           uint32_t* out_broken) {
    clear_error();
    if (!s || !cfg) {
        set_error("vx_fracture_commit: null argument");
        return VX_BAD_INPUT;
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) {
        set_error("vx_fracture_commit: invalid dt=%g", dt);
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    return fracture_stage(s, dt, cfg, out, out_broken);
}

int32_t vx_scene_get_bond_state(vx_scene* s, float* plastic, float* damage, float* eqp, float* fatigue) {
    clear_error();
    if (!s) return VX_BAD_INPUT;
    cudaSetDevice(s->device);
    const size_t m = 3 * (size_t)s->n;
    std::vector<float4> a(m), b(m), c(m);
    if (m) {
        VX_TRY(cudaMemcpyAsync(a.data(), s->bond_a, m * sizeof(float4), cudaMemcpyDeviceToHost, s->stream), "bonds");
        VX_TRY(cudaMemcpyAsync(b.data(), s->bond_b, m * sizeof(float4), cudaMemcpyDeviceToHost, s->stream), "bonds");
        VX_TRY(cudaMemcpyAsync(c.data(), s->bond_c, m * sizeof(float4), cudaMemcpyDeviceToHost, s->stream), "bonds");
        VX_TRY(cudaStreamSynchronize(s->stream), "bonds");
    }
    for (size_t e = 0; e < m; ++e) {
        if (plastic) plastic[3 * e] = b[e].x, plastic[3 * e + 1] = b[e].y, plastic[3 * e + 2] = b[e].z;
        if (damage) damage[e] = a[e].w;
        if (eqp) eqp[e] = b[e].w;
        if (fatigue) fatigue[e] = c[e].y;
    }
    return VX_OK;
}

int32_t vx_scene_get_last_forces(vx_scene* s, float* force) {
    VX_CHECK_SCENE(s, force);
    const size_t m = 9 * (size_t)s->n;
    if (m) {
        VX_TRY(cudaMemcpyAsync(force, s->last_force, m * sizeof(float), cudaMemcpyDeviceToHost, s->stream), "forces");
        VX_TRY(cudaStreamSynchronize(s->stream), "forces");
    }
    return VX_OK;
}

int32_t vx_scene_checkpoint(vx_scene* s, int32_t op) {
    clear_error();
    if (!s || (op != 0 && op != 1)) {
        set_error("vx_scene_checkpoint: bad argument");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    size_t n = s->n;
    if (op == 0) {
        VX_TRY(cudaMemcpyAsync(s->save_pos, s->pos, 3 * n * 8, cudaMemcpyDeviceToDevice, s->stream), "checkpoint");
        VX_TRY(cudaMemcpyAsync(s->save_rot, s->rot, n * sizeof(double4), cudaMemcpyDeviceToDevice, s->stream),
               "checkpoint");
    } else {
        VX_TRY(cudaMemcpyAsync(s->pos, s->save_pos, 3 * n * 8, cudaMemcpyDeviceToDevice, s->stream), "restore");
        VX_TRY(cudaMemcpyAsync(s->rot, s->save_rot, n * sizeof(double4), cudaMemcpyDeviceToDevice, s->stream),
               "restore");
    }
    return VX_OK;
}

void* vx_scene_stream(vx_scene* s) { return s ? (void*)s->stream : nullptr; }

// One cache line per choice: "<gpu> <sms> <precision> <log2 n> <kernel> <blocks> <us>".
static std::string tune_key(vx_scene* s, int32_t precision) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, s->device);
    std::string name = prop.name;
    for (char& c : name)
        if (c == ' ' || c == '\t') c = '_';
    int bucket = 0;
    for (uint32_t v = s->n; v > 1; v >>= 1) ++bucket;
    char buf[256];
    snprintf(buf, sizeof buf, "%s %d %d %d", name.c_str(), s->sm_count, precision, bucket);
    return buf;
}

int32_t vx_scene_autotune(vx_scene* s, int32_t precision, const char* cache_path, vx_tune_result* out) {
    clear_error();
    if (!s || !out || (precision != VX_PRECISION_FP64 && precision != VX_PRECISION_MIXED)) {
        set_error("vx_scene_autotune: bad argument");
        return VX_BAD_INPUT;
    }
    if (!s->assembled || s->n == 0) {
        set_error("vx_scene_autotune: run a pass first (the tuner times the assembled system)");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    std::memset(out, 0, sizeof *out);
    const std::string key = tune_key(s, precision);
    std::vector<std::string> lines;
    if (cache_path) {
        if (FILE* f = std::fopen(cache_path, "r")) {
            char line[512];
            while (std::fgets(line, sizeof line, f)) {
                std::string l(line);
                while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
                if (l.empty()) continue;
                if (l.compare(0, key.size() + 1, key + " ") == 0) {
                    int kernel = 0, blocks = 0;
                    double us = 0.0;
                    bool usable = false;
                    if (std::sscanf(l.c_str() + key.size() + 1, "%d %d %lf", &kernel, &blocks, &us) == 3) {
                        if (kernel == VX_KERNEL_STREAMING) {
                            usable = blocks >= 3 && blocks <= 5;
                        } else if (kernel == VX_KERNEL_PERSISTENT && blocks >= VX_PERSIST_BRICK_T1_256 &&
                                   blocks <= VX_PERSIST_RANGE_896) {
                            const int old_form = s->persist_form;
                            apply_tuning(s, kernel, blocks);
                            usable = persistent_plan(s);
                            if (!usable) apply_tuning(s, s->tuned_kernel, old_form);
                        }
                    }
                    if (usable) {
                        std::fclose(f);
                        apply_tuning(s, kernel, blocks);
                        out->kernel = kernel;
                        out->blocks_per_sm = blocks;
                        out->us_per_iteration = us;
                        out->from_cache = 1;
                        return VX_OK;
                    }
                    continue;  // a stale entry for this key is dropped
                }
                lines.push_back(l);
            }
            std::fclose(f);
        }
    }
    struct Cand {
        int32_t kernel;
        int blocks;
    };
    std::vector<Cand> cands = {{VX_KERNEL_STREAMING, 3}, {VX_KERNEL_STREAMING, 4}, {VX_KERNEL_STREAMING, 5}};
    const int old_blocks = s->pcg_minb, old_form = s->persist_form;
    if (precision == VX_PRECISION_MIXED) {
        // the persistent forms that fit; brick forms with the same blocks and
        // threads per REV (a large scene reaches the same tiles from either
        // minimum) are timed once
        std::vector<std::array<unsigned, 3>> seen;
        for (int form = VX_PERSIST_BRICK_T1_256; form <= VX_PERSIST_RANGE_896; ++form) {
            s->persist_form = form;
            s->persist_checked = false;
            if (!persistent_plan(s)) continue;
            if (form < VX_PERSIST_RANGE) {
                const std::array<unsigned, 3> shape = {s->brick_G, s->brick_cap, s->brick_tpr};
                if (std::find(seen.begin(), seen.end(), shape) != seen.end()) continue;
                seen.push_back(shape);
            }
            cands.push_back({VX_KERNEL_PERSISTENT, form});
        }
        s->persist_form = old_form;
        s->persist_checked = false;
    }
    int best = -1;
    for (size_t k = 0; k < cands.size() && k < 12; ++k) {
        double us = 0.0;
        int32_t r = time_candidate(s, precision, cands[k].kernel, cands[k].blocks, &us);
        if (r != VX_OK) {
            s->persist_form = old_form;
            s->persist_checked = false;
            apply_tuning(s, -1, old_blocks);
            return r;
        }
        out->candidate_kernel[k] = cands[k].kernel;
        out->candidate_blocks[k] = cands[k].blocks;
        out->candidate_us[k] = us;
        out->candidates = (uint32_t)(k + 1);
        if (best < 0 || us < out->candidate_us[best]) best = (int)k;
    }
    if (cands[best].kernel != VX_KERNEL_PERSISTENT) {
        s->persist_form = old_form;
        s->persist_checked = false;
    }
    apply_tuning(s, cands[best].kernel, cands[best].blocks);
    out->kernel = cands[best].kernel;
    out->blocks_per_sm = cands[best].blocks;
    out->us_per_iteration = out->candidate_us[best];
    if (cache_path) {
        if (FILE* f = std::fopen(cache_path, "w")) {
            for (const std::string& l : lines) std::fprintf(f, "%s\n", l.c_str());
            std::fprintf(f, "%s %d %d %.3f\n", key.c_str(), out->kernel, out->blocks_per_sm, out->us_per_iteration);
            std::fclose(f);
        } else {
            set_error("vx_scene_autotune: cannot write %s (the choice is applied, not stored)", cache_path);
        }
    }
    return VX_OK;
}

int32_t vx_scene_kernel_times(vx_scene* s, int32_t precision, uint32_t reps, void* flush, uint64_t flush_bytes,
                              double* out_us) {
    clear_error();
    if (!s || !out_us || reps == 0) {
        set_error("vx_scene_kernel_times: bad argument");
        return VX_BAD_INPUT;
    }
    if (!s->assembled) {
        set_error("vx_scene_kernel_times: no assembled system");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    return kernel_times(s, precision, reps, flush, flush_bytes, out_us);
}

}  // extern "C"
