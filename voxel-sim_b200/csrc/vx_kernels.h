// vx_kernels.h — launchers of the corotational-solve kernels.
#pragma once

#include "vx_internal.h"

namespace vx {

// Plain-pointer view of a scene passed by value to kernels.
struct SceneView {
    uint32_t n;
    const double* pos;
    const double* pred;
    const double* loads;
    const double4* rot;
    const uint8_t* kin;
    const uint8_t* flags;
    const float4* param0;
    const float4* param1;
    const uint32_t* matid;
    const vx_material* materials;
    const uint32_t* nbr;
    const uint32_t* rev;
    const float4* bond_a;
    const float4* bond_b;
    const uint8_t* tile_on;  // per 256-REV tile: 0 = skip (pool tiles of disabled or free slots); null = all on
    const uint32_t* tile_scene;  // per tile: pool slot (for per-slot maxima); null for a single scene
};

__device__ __forceinline__ bool tile_active(const uint8_t* tile_on, size_t i) {
    return tile_on == nullptr || tile_on[i >> 8] != 0;
}

SceneView view_of(const vx_scene* s);

// free-axis flags from kinematic flags and target masks
cudaError_t launch_flags(vx_scene* s);
// reverse neighbour table rev[a][j] = i where nbr[a][i] == j
cudaError_t launch_reverse_neighbors(vx_scene* s);
// dense-grid topology build (vx_build_topology)
cudaError_t launch_topology(const int32_t* d_cells, const uint8_t* d_kin, uint32_t n, const int32_t* lo,
                            const int32_t* ext, int32_t* d_grid, uint32_t* d_nbr, uint32_t* d_dup,
                            cudaStream_t stream);
// polar-decomposition rotation fit; writes the max angle bits to s->max_angle_bits
cudaError_t launch_fit_rotations(vx_scene* s);
// bond and REV assembly of one pass (h = substep)
cudaError_t launch_assembly(vx_scene* s, double h, bool reuse_preconditioner);
// x += dx for active axes
cudaError_t launch_apply_correction(vx_scene* s);
// substep prediction and velocity update of the fixed step (vx_step.cu)
cudaError_t launch_predict(vx_scene* s, const double* gravity, double h);
cudaError_t launch_advance_targets(vx_scene* s, const double* d_delta);
cudaError_t launch_velocity(vx_scene* s, double h);
cudaError_t launch_velocity_update(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* d_value,
                                   int32_t op);
cudaError_t launch_gather3(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* field, double* d_out);
cudaError_t launch_scatter3(vx_scene* s, uint32_t count, const uint32_t* d_index, const double* d_value,
                            double* field);
// connected components of the bond graph with the reference's cluster numbering (vx_clusters.cu)
// collision::project and resolve_velocities_with_precontact (vx_contact.cu)
int32_t contact_project(vx_scene* s, vx_contact_stats* out, uint32_t* slot_contacts);
int32_t contact_resolve(vx_scene* s, const double* pre_contact, double restitution, double friction,
                        vx_contact_heat* out);
uint32_t contact_count(const vx_scene* s);
uint64_t contact_state_bytes(uint32_t n);
int32_t pool_stream_priority(vx_pool* p, int priority);
void contact_release(vx_scene* s);
cudaError_t launch_rest_positions(vx_scene* s);
cudaError_t launch_rest_range(vx_scene* s, size_t first, size_t count);

cudaError_t launch_rebuild_clusters(vx_scene* s);
uint32_t cluster_scan_blocks(uint32_t n);
// fracture stage: fracture::update on every bond of the last assembly (dt = substep)
cudaError_t launch_fracture_commit(vx_scene* s, double dt, const vx_fracture_config* cfg);
// fracture stage plus the reverse-table rebuild when bonds broke (vx_capi.cu)
int32_t fracture_stage(vx_scene* s, double dt, const vx_fracture_config* cfg, vx_dissipation* out,
                       uint32_t* out_broken);
// bond stress / ratio / force
cudaError_t launch_bond_stress(vx_scene* s, float* d_ratio, float* d_force, uint32_t* d_near, uint32_t cap);

// PCG drivers (vx_pcg.cu)
int32_t solve_fp64(vx_scene* s, double tolerance, uint32_t max_iterations, vx_pass_stats* out);
int32_t solve_mixed(vx_scene* s, double tolerance, uint32_t max_iterations, double inner_tolerance,
                    uint32_t max_outer, int32_t kernel, vx_pass_stats* out);
// persistent on-chip FP32 inner solve (vx_persistent.cu)
bool persistent_plan(vx_scene* s);
int32_t solve_inner_persistent(vx_scene* s, double tolerance, uint32_t max_iterations);
bool brick_plan(vx_scene* s, int form);
bool expanded_plan(vx_scene* s);
int32_t solve_inner_expanded(vx_scene* s, double tolerance, uint32_t max_iterations);
int32_t solve_inner_slots_expanded(vx_scene* s, const uint4* d_blocks, SlotState* st, unsigned G, uint32_t cap);
bool neighbor_deltas_fit(vx_scene* s);
uint32_t persistent_block_cap();
int32_t solve_inner_slots(vx_scene* s, const uint4* d_blocks, SlotState* st, unsigned G, uint32_t cap);
int32_t solve_inner_brick(vx_scene* s, double tolerance, uint32_t max_iterations);
// |b - A x64| / |b| with the FP64 operator (device scalars updated)
int32_t true_residual(vx_scene* s, double* out);
// autotuning: time one candidate (microseconds per inner iteration) and apply a choice (vx_pcg.cu)
int32_t time_candidate(vx_scene* s, int32_t precision, int32_t kernel, int mb, double* us);
void apply_tuning(vx_scene* s, int32_t kernel, int mb);
// CUDA-event timing of the matvec and update kernels (microseconds per launch)
int32_t kernel_times(vx_scene* s, int32_t precision, uint32_t reps, void* flush, uint64_t flush_bytes,
                     double* out_us);

}  // namespace vx
