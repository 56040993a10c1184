// vx_internal.h — host-side structures behind the C ABI (include/vxcorot.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/vxcorot.h"

namespace vx {

struct ContactState;  // grow-only buffers of the contact stage (vx_contact.cu)

// Thread-local error message returned by vx_last_error().
void set_error(const char* fmt, ...);
void clear_error();

// Per-slot device state of a pool pass (vx_pool.cu; the persistent inner solve
// of vx_persistent.cu reads a slot's inner target and writes its outcome).
struct SlotState {
    // FP32 inner solve
    double rz, initial, beta, alpha, residual_in, tol_in;
    uint32_t its, max_its;
    int32_t done, status_in;
    // FP64 refinement
    double r64_norm, b_norm, residual;
    uint32_t used, outer;
    int32_t status, outer_done;
    int32_t inner_on, enabled;
};

// Device-side recurrence scalars of one PCG solve (FP64 or FP32 inner).
struct PcgScalars {
    double rz[2];       // r . z of iteration k in slot k & 1
    double pap;         // p . Ap
    double rr;          // r . r
    double initial;     // |r0|
    double alpha;
    double beta;
    double residual;    // |r| / |r0|
    double tolerance;   // stop when residual < tolerance
    double b_norm;      // |b| (outer FP64 residual)
    double r64_norm;    // |b - A x| (outer)
    uint32_t max_iterations;
    uint32_t iterations;
    int32_t done;       // 1 = stop issuing work
    int32_t status;     // VX_OK, VX_NOT_CONVERGED, VX_NONFINITE
    uint32_t counter[4];  // last-block tickets of the fused reductions
};

// Per-bond storage of the last assembly (SoA, bond e = axis * n + i).
struct BondArrays {
    double* k64;        // [18][n]  world K (sym6) per axis, 0 if not assembled
    float* k32;         // [3][6][kstride32(n)]: FP32 copy, axis-padded to 16 bytes
    double* mat_k;      // [6][3n]  undamaged local K (sym6) for stress
    double4* frame_q;   // [3n]     bond frame quaternion (slerp midpoint)
    double* force;      // [3][3n]  K (x_j - x_i - rest) of assembled bonds
    uint8_t* state;     // [3n]     0 none, 1 fracture only, 2 assembled
};

struct Arena {
    char* base = nullptr;
    size_t size = 0;
    size_t used = 0;
    template <typename T>
    T* take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

}  // namespace vx

struct vx_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
};

struct vx_scene {
    vx_ctx* ctx = nullptr;        // creating context (not dereferenced after creation)
    int device = 0;               // the scene's GPU; the scene may outlive its context
    uint32_t n = 0;
    uint32_t blocks = 0;          // grid of the per-REV kernels (256 threads)
    cudaStream_t stream = nullptr;
    vx::Arena arena;

    // REV state
    double* pos;                  // [3][n]
    double* pred;                 // [3][n]
    double* loads;                // [3][n]
    double* target;               // [3][n]
    double4* rot;                 // [n]
    uint8_t* kin;                 // [n]
    uint8_t* tmask;               // [n]
    uint8_t* flags;               // [n] free axes (bit a)
    float4* param0;               // [n] fibre xyz, anisotropy
    float4* param1;               // [n] solid, thermal strength, thermal delta, mass
    uint32_t* matid;              // [n]
    vx_material* materials;       // [material_count]
    uint32_t material_count;
    uint32_t* nbr;                // [3][n]
    uint32_t* rev;                // [3][n]
    float4* bond_a;               // [3n] formation xyz, damage
    float4* bond_b;               // [3n] plastic xyz, equivalent plastic strain
    float4* bond_c;               // [3n] plastic work, fatigue damage, previous / reversal stress ratio
    float* bond_d;                // [3n] loading increment (fatigue)
    float* last_force;            // [3n][3] Bond workspace last_force, N, of the last fracture commit
    double* frac_partials;        // [5 * 3 * blocks] block partials of the dissipation
    double* frac_totals;          // [8] dissipation totals of the last fracture stage
    uint32_t* frac_counter;       // [2] last-block ticket, bonds broken
    uint32_t* clusters;           // [n] cluster id per REV (VX_EMPTY for kinematic REVs)
    uint32_t* cl_parent;          // [n] union-find parents
    uint32_t* cl_root;            // [n] component root (smallest REV)
    uint32_t* cl_first;           // [n] per root: first non-kinematic REV
    uint32_t* cl_scan;            // [n] exclusive scan of first-REV flags within a scan block
    uint32_t* cl_bsum;            // [n / 1024 + 2] scan-block totals, then the cluster count
    uint32_t* cl_err;             // [1] a union exceeded its retry bound

    vx::BondArrays bonds;

    // assembled system
    double* d64;                  // [6][n] projected diagonal block
    double* dinv64;               // [6][n]
    float* d32;
    float* mh2_32;  // [n] m/h^2 of the last assembly: the FP32 operator's mass term
    float* dinv32;
    double* b64;                  // [3][n]

    // solver vectors
    double* x64;                  // [3][n] correction dx
    double* r64;
    double* z64;
    double* p64[2];
    double* ap64;
    float* x32;
    float* r32;
    float* z32;
    float* p32[2];
    float* ap32;
    double* vel;                  // [3][n] velocity, m/s (Voxel::velocity)
    double* prev;                 // [3][n] positions at the start of the substep (Scene::previous)
    double* drift;                // [3][n] predicted velocity of the substep (drift_velocity)
    float* rest;                  // [3][n] creation positions (Scene::rest_positions)
    vx::ContactState* contact = nullptr;  // allocated by the first contact call
    double* save_pos;             // [3][n] checkpoint
    double4* save_rot;            // [n]
    float* out_ratio;             // [3n] bond stress outputs
    float* out_force;             // [9n]
    uint32_t* out_near;           // [3n]
    double* partials;             // [4 * blocks]: p.Ap partials, then r.z / r.r partials
    vx::PcgScalars* sc;           // device scalars (FP64 solve / outer)
    vx::PcgScalars* sc32;         // device scalars (FP32 inner solve)
    unsigned long long* max_angle_bits;
    uint32_t* near_count;
    uint32_t* bond_count;         // bonds assembled by the last pass
    unsigned* barrier;            // [4] persistent kernel: u64 arrival count, error flag, pad
    float* zp32;                  // [6n] persistent kernel's published (z, p_old): float4[n] then float2[n]
    uint32_t* nbcode;             // [3][n] neighbour deltas j - i as int16 pairs (0 = none): own x|y, own z|rev x, rev y|z
    uint32_t* nbcode_bad;         // [1] neighbour entries a delta cannot encode

    // host mirrors
    double* h_stage = nullptr;       // pinned staging of host copies [4 * stage_revs doubles]
    size_t stage_revs = 0;           // n for a single scene; capped for pools
    vx::PcgScalars* h_sc = nullptr;  // pinned
    int32_t* h_done = nullptr;       // pinned [2]
    cudaEvent_t ev[2] = {nullptr, nullptr};

    // cached CUDA graphs of PCG iteration chunks
    cudaGraphExec_t chunk64 = nullptr;
    cudaGraphExec_t chunk32 = nullptr;

    // scene pool: several scenes in tile-aligned ranges of one arena (pool_slots > 0)
    uint32_t pool_slots = 0;      // slot capacity; 0 = a single scene
    uint8_t* tile_on = nullptr;   // [tiles] 1 = tile of a slot taking part in the current call
    uint32_t* tile_scene = nullptr;  // [tiles] slot of the tile, VX_EMPTY when free
    uint32_t* pool_slot_first = nullptr;  // [pool_slots] first tile of each slot (device)
    uint32_t* pool_slot_revs = nullptr;   // [pool_slots] REVs of each slot (device)
    uint32_t launches = 0;        // kernels launched by the current pass
    int sm_count = 148;           // SMs of the scene's GPU
    unsigned grid32 = 0;          // grid of the FP32 / FP64 PCG kernels (0 = not yet chosen)
    int pcg_minb = 4;             // register budget of the streaming kernels: blocks per SM (3, 4 or 5)
    int tuned_kernel = -1;        // inner kernel chosen by the autotuner (-1 = none)
    unsigned grid64 = 0;
    // persistent (on-chip) inner solve plan
    bool persist_checked = false;
    bool persist_ok = false;
    unsigned persist_G = 0, persist_cap = 0, persist_R = 0, persist_T = 512;
    size_t persist_smem = 0;
    int nbcode_state = 0;         // 0 = not yet read back, 1 = all deltas encoded, 2 = some did not fit
    // brick plan of the on-chip inner solve (vx_brick.cu): blocks own spatially
    // compact sets of REVs; one device allocation holds the plan's tables
    bool brick_ok = false;
    unsigned brick_G = 0, brick_cap = 0, brick_hz = 0, brick_hk = 0, brick_R = 0, brick_tpr = 1;
    int persist_form = 0;             // 0: the range plan, else the brick plan (1 thread per REV, >= 256
                                      // REVs per block); VX_PERSIST_*: that form only (the autotuner's choice)
    size_t brick_smem = 0;
    void* brick_buf = nullptr;
    uint4* brick_info = nullptr;      // [G] own REVs, halo z slots, halo K slots, neighbour blocks
    uint32_t* brick_own = nullptr;    // [G][cap] REV of each local REV
    uint32_t* brick_ref = nullptr;    // [G][3][cap] six 16-bit neighbour refs per local REV
    uint32_t* brick_hzg = nullptr;    // [G][hz] REV of each halo z slot
    uint32_t* brick_hke = nullptr;    // [G][hk] bond of each halo K slot
    uint32_t* brick_nbk = nullptr;    // [G][32] blocks whose REVs are in the halo
    uint32_t* brick_pub = nullptr;    // [G] iteration whose z the block has published
    double* brick_part = nullptr;     // [3][G] grid-reduction partials
    // range plan with one reduction per iteration (vx_expanded.cu): published
    // triples (u, v, p) in two parities and the partials, one allocation
    bool exp_ok = false;
    unsigned exp_G = 0, exp_cap = 0, exp_R = 0;
    size_t exp_smem = 0;
    void* exp_buf = nullptr;
    float4* exp_pa = nullptr;         // [2][n] (u, v.x)
    float4* exp_pb = nullptr;         // [2][n] (v.y, v.z, p.x, p.y)
    float* exp_pc = nullptr;          // [2][n] p.z
    double* exp_part = nullptr;       // [14][G]
    uint32_t active = 0;          // REVs with a free axis (cached per target set)
    bool active_cached = false;
    bool assembled = false;
    bool have_dinv = false;
};

namespace vx {
uint64_t scene_bytes(uint32_t n, uint32_t material_count);
}
