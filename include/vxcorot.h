/*
 * vxcorot.h — C ABI of the B200 corotational elastic solve.
 *
 * This is the drop-in boundary for the Voxel-sim solver (TheLastie/Voxel-sim).
 * In the reference, control crosses to the GPU in one place,
 * `cuda_solver::solve_pcg` (src/cuda_solver.rs:301-309), called from
 * `solve_coupled` (src/solver.rs:1778-1786). Everything else on the hot path
 * (rotation fit, bond assembly, bond stress) runs on the host there. Here every
 * part of the path has an entry point:
 *
 *   vx_solve_pcg_f32            replaces cuda_solver::solve_pcg (same arguments,
 *                               same layouts, same convergence rule)
 *   vx_fit_rotations            replaces solver::fit_rotations (src/solver.rs:327-417)
 *   vx_corotational_pass        replaces solver::solve_coupled (src/solver.rs:1542-1929):
 *                               assembly (make_constraint, :1325-1345), RHS/diagonal
 *                               (:1576-1636), block-Jacobi PCG (:1833-1911),
 *                               position update (:1921-1923)
 *   vx_bond_stress              replaces the stress/limit part of the fracture loop
 *                               (src/solver.rs:627-665 -> bond_limits :124-158 ->
 *                               fracture::pair_limits / update, src/fracture.rs:76-133,
 *                               :210-292)
 *
 * Conventions
 *   - Every function returns an int32_t status (VX_OK = 0). No exception crosses
 *     the boundary. vx_last_error() returns a thread-local message that names
 *     the failing operation, like the reference's Err(String).
 *   - Host pointers are borrowed for the duration of the call only.
 *   - Vectors are xyz-interleaved (3 values per REV, like glam::Vec3 slices);
 *     quaternions are xyzw (glam::Quat); 3x3 matrices are row-major, which is
 *     the packing of src/solver.rs:1741-1751.
 *   - Per-bond arrays are axis-major: bond (axis, i) is element axis*n + i, the
 *     layout of Scene::bonds (src/scene.rs:322), whose owner is the lower
 *     endpoint i and whose partner is neighbor[axis*n + i] (the +axis cell).
 *   - VX_EMPTY (u32::MAX, src/bond.rs:2) marks a missing neighbour.
 *   - A scene handle is single-threaded: calls on one handle must not overlap.
 */
#ifndef VXCOROT_H
#define VXCOROT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_EMPTY 0xFFFFFFFFu
#define VX_ABI_VERSION 1

/* Status codes. */
enum {
    VX_OK = 0,
    VX_NOT_CONVERGED = 1, /* iteration cap reached above tolerance (outputs still written) */
    VX_NONFINITE = 2,     /* NaN/Inf in an input or produced by the solve */
    VX_OOM = 3,           /* device allocation failed or admission refused */
    VX_BAD_INPUT = 4,     /* invalid argument (null pointer, size, index) */
    VX_CUDA_ERROR = 5,    /* a CUDA runtime call failed */
    VX_TIMEOUT = 6,       /* a bounded device-side wait ran out */
    VX_NO_DEVICE = 7      /* no CUDA device, or the device was lost */
};

/* Fracture modes, src/material.rs:3-8. */
enum { VX_BRITTLE = 0, VX_DUCTILE = 1, VX_MIXED = 2 };

/* Kernel choice for the FP32 inner solve of the MIXED form. */
enum {
    VX_KERNEL_AUTO = 0,       /* persistent when the scene fits on chip, else streaming */
    VX_KERNEL_STREAMING = 1,  /* two grid-stride kernels per iteration, replayed as CUDA graphs */
    VX_KERNEL_PERSISTENT = 2  /* one cooperative kernel per inner solve, state in shared memory */
};

/* Precision forms of a corotational pass. */
enum {
    VX_PRECISION_FP64 = 0,  /* plain FP64 block-Jacobi PCG */
    VX_PRECISION_MIXED = 1  /* FP32 inner PCG inside FP64 iterative refinement */
};

/*
 * Material fields read by the stiffness and limit laws: the subset of
 * material::Material (src/material.rs:20-63) that tensor_compliance
 * (src/solver.rs:37-63), bond_thermal_rest (:78-95) and pair_limits
 * (src/fracture.rs:76-133) use. Values are the f32 values of the reference.
 */
typedef struct vx_material {
    float density;
    float young;
    float young_perp;
    float shear;
    float tensile_strength;
    float tensile_strength_perp;
    float compressive_strength;
    float compressive_strength_perp;
    float shear_strength;
    float shear_strength_perp;
    float yield_strength;
    float hardening_modulus;
    float failure_plastic_strain;
    float fracture_energy;
    float fracture_energy_perp;
    float thermal_expansion_parallel;
    float thermal_expansion_perpendicular;
    int32_t fracture_mode; /* VX_BRITTLE / VX_DUCTILE / VX_MIXED */
} vx_material;

/*
 * One scene (a REV lattice). Mirrors the fields of Scene (src/scene.rs:309-351)
 * and Voxel (src/voxel.rs:7-21) that the elastic solve reads. Phase-dependent
 * values (solid fraction, pre-melt strength scale, temperature change since
 * creation) are derived by the host from its thermal state, as
 * Material::phase_state / thermal_strength_scale do (src/material.rs:485-565).
 * Optional arrays may be NULL (then zero, or one for solid/thermal_strength).
 */
typedef struct vx_scene_desc {
    uint32_t n;                       /* REV count */
    const double* position;           /* 3n, metres */
    const double* rotation;           /* 4n xyzw, or NULL = identity */
    const uint8_t* kinematic;         /* n, Voxel::kinematic */
    const float* mass;                /* n, kg (density * CELL^3) */
    const uint32_t* material;         /* n, index into materials */
    const vx_material* materials;
    uint32_t material_count;
    const float* fiber;               /* 3n, Microstructure::fibers() = orientation * Z */
    const float* anisotropy;          /* n, Microstructure::anisotropy */
    const float* solid_fraction;      /* n or NULL (1) */
    const float* thermal_strength;    /* n or NULL (1) */
    const float* thermal_delta;       /* n or NULL (0): T - T_reference, kelvin */
    const uint32_t* neighbor;         /* 3n axis-major, Bond::neighbor */
    const float* formation_offset;    /* 9n ((axis*n+i)*3+c) or NULL */
    const float* plastic_strain;      /* 9n or NULL */
    const float* damage;              /* 3n or NULL */
} vx_scene_desc;

/* Parameters of one corotational pass (one call of solve_coupled). */
typedef struct vx_pass_params {
    double h;                    /* substep length, s (fixed_dt / substeps, src/solver.rs:475) */
    double tolerance;            /* relative residual target */
    uint32_t max_iterations;     /* PCG iteration cap (inner iterations for MIXED) */
    int32_t precision;           /* VX_PRECISION_FP64 or VX_PRECISION_MIXED */
    int32_t reuse_preconditioner;/* 1: keep the block-Jacobi inverse of the previous pass
                                    (CPU path, src/solver.rs:554 and :1639) */
    double inner_tolerance;      /* MIXED only: relative target of each FP32 inner solve
                                    (0 = default 1e-5) */
    uint32_t max_outer;          /* MIXED only: refinement cap (0 = default 30) */
    int32_t kernel;              /* MIXED only: VX_KERNEL_AUTO / _STREAMING / _PERSISTENT */
} vx_pass_params;

typedef struct vx_pass_stats {
    uint32_t iterations;         /* PCG iterations (FP32 inner iterations for MIXED) */
    uint32_t outer_iterations;   /* FP64 refinement steps (MIXED), else 1 */
    double residual;             /* recursive relative residual |r|/|r0| (FP64 form), as
                                    Scene::solver_residual (src/solver.rs:1882) */
    double true_residual;        /* |b - A dx|/|b| recomputed in FP64 with the FP64 operator */
    uint32_t active;             /* REVs with at least one free axis */
    uint32_t bonds_assembled;    /* bonds that entered the system */
    int32_t converged;
    uint32_t kernel_launches;    /* kernels this pass launched (early-exit ones included) */
} vx_pass_stats;

/* Last error message of the calling thread ("" when none). */
const char* vx_last_error(void);
int32_t vx_abi_version(void);

/*
 * Compatibility shim: the exact contract of cuda_solver::solve_pcg
 * (src/cuda_solver.rs:301-501). Inputs are the engine's packed active-REV
 * system (src/solver.rs:1731-1777): rhs[3n], neighbors[6n] (VX_EMPTY = unused
 * slot), diagonal[9n], blocks[54n] (six row-major 3x3 off-diagonal blocks per
 * row), inverse_diagonal[9n]. Block-Jacobi PCG with f32 vectors, f64 dot
 * accumulation and f32 alpha/beta; the residual |r|/|b| is checked every 16
 * iterations and at the cap, converging when <= tolerance. Returns VX_OK with
 * out_dx[3n] written, or VX_NOT_CONVERGED / VX_NONFINITE (out_dx still written)
 * where the reference returns Err and the engine falls back.
 */
int32_t vx_solve_pcg_f32(const float* rhs, const uint32_t* neighbors, const float* diagonal,
                         const float* blocks, const float* inverse_diagonal, uint32_t n,
                         uint32_t max_iterations, float tolerance, float* out_dx,
                         uint32_t* out_iterations, float* out_relative);

/*
 * vx_solve_pcg_f32_noalloc — no counterpart in the reference.
 *
 * The same solve as vx_solve_pcg_f32 for callers that cannot allocate device
 * memory: an engine that sizes and owns every byte of its GPU up front (a
 * fixed per-GPU budget, as an admission-controlled server keeps), or a step
 * loop in which a cudaMalloc/cudaFree, which can block on the device, is not
 * acceptable. The caller passes device pointers: the packed system in the
 * layouts of vx_solve_pcg_f32 and d_out_dx[3n] for the correction.
 * out_iterations and out_relative are host pointers (or NULL); stream is a
 * cudaStream_t (NULL = the legacy default stream). The function calls no
 * cudaMalloc, cudaFree or other allocating routine: its work vectors,
 * reduction partials and scalars live in one fixed device array of
 * VX_NOALLOC_SCRATCH_BYTES that every GPU which loads this library keeps until
 * the process exits. Systems of more than VX_NOALLOC_MAX_ROWS rows are
 * rejected with VX_BAD_INPUT.
 *
 * Every call looks up that array's device address on the current device
 * (cudaGetSymbolAddress), so a device reset in between is harmless. Every call
 * also reads its convergence scalars back and synchronizes its stream, so it
 * must never be called while that stream is being captured into a graph. All
 * calls share the one array and each call starts by clearing the parts that
 * must be zero; calls that overlap on the GPU (other threads or streams on the
 * same device) race on it and must not run at the same time. The initial
 * residual norm is summed in the same order as vx_solve_pcg_f32 sums it, so the
 * two entry points stop at the same iteration on the same system.
 */
#define VX_NOALLOC_MAX_ROWS 65536u
#define VX_NOALLOC_SCRATCH_BYTES 4194304u
int32_t vx_solve_pcg_f32_noalloc(const float* d_rhs, const uint32_t* d_neighbors, const float* d_diagonal,
                                 const float* d_blocks, const float* d_inverse_diagonal, uint32_t n,
                                 uint32_t max_iterations, float tolerance, float* d_out_dx,
                                 uint32_t* out_iterations, float* out_relative, void* stream);

/* Device context (one per GPU and host thread of control). */
typedef struct vx_ctx vx_ctx;
typedef struct vx_scene vx_scene;

int32_t vx_ctx_create(int32_t device, vx_ctx** out_ctx);
int32_t vx_ctx_destroy(vx_ctx* ctx);

/*
 * Bond topology from lattice cells, on the device: for each REV i and axis,
 * neighbor[axis*n+i] = the REV at cell + e_axis when both have the same
 * kinematic flag, else VX_EMPTY. Same indices as Scene::from_voxels
 * (src/scene.rs:558-570) and Scene::new (:1668-1681). cells[3n] are integer
 * lattice coordinates and must be unique.
 */
int32_t vx_build_topology(vx_ctx* ctx, const int32_t* cells, const uint8_t* kinematic,
                          uint32_t n, uint32_t* out_neighbor);

int32_t vx_scene_create(vx_ctx* ctx, const vx_scene_desc* desc, vx_scene** out_scene);
int32_t vx_scene_destroy(vx_scene* scene);
/* Device bytes held by a scene of n REVs (admission estimate). */
uint64_t vx_scene_footprint_bytes(uint32_t n);

int32_t vx_scene_set_positions(vx_scene* scene, const double* xyz);
int32_t vx_scene_get_positions(vx_scene* scene, double* xyz);
int32_t vx_scene_set_rotations(vx_scene* scene, const double* xyzw);
int32_t vx_scene_get_rotations(vx_scene* scene, double* xyzw);
/*
 * Axis targets of this substep (the merged persistent + per-step targets of
 * src/solver.rs:449-460). mask[i] bit a set = axis a of REV i is targeted;
 * a targeted axis leaves the PCG system (free = 0, src/solver.rs:1554-1565).
 * xyz may be NULL when only the mask matters.
 */
int32_t vx_scene_set_targets(vx_scene* scene, const uint8_t* mask, const double* xyz);
/* Applied nodal loads in newtons (applied_loads, src/solver.rs:461-474). */
int32_t vx_scene_set_loads(vx_scene* scene, const double* xyz);
/* Predicted positions of this substep (src/solver.rs:542); NULL = current positions. */
int32_t vx_scene_set_predicted(vx_scene* scene, const double* xyz);
/* Bond state written by fracture (neighbor, plastic strain, damage, formation offset). */
int32_t vx_scene_set_bonds(vx_scene* scene, const uint32_t* neighbor, const float* plastic_strain,
                           const float* damage, const float* formation_offset);
int32_t vx_scene_get_neighbors(vx_scene* scene, uint32_t* neighbor);

/* Polar-decomposition rotation fit; returns the largest angle change (rad). */
int32_t vx_fit_rotations(vx_scene* scene, double* out_max_angle);

/* One corotational pass: assemble, solve, x += dx. */
int32_t vx_corotational_pass(vx_scene* scene, const vx_pass_params* params, vx_pass_stats* out);

/*
 * Stress ratio of every bond against its directional limits, evaluated with
 * the frames and undamaged stiffness of the last pass and the current
 * rotations and positions (src/solver.rs:627-647). ratio[3n] (axis-major);
 * -1 where the fracture loop skips the bond (no neighbour, kinematic owner,
 * or not part of the last assembly). Bonds with |ratio - 1| <= 1e-6 are
 * listed in near[] (bond index axis*n+i, at most cap) and counted in
 * *near_count. force[9n] (or NULL) receives Bond workspace last_force, N.
 */
int32_t vx_bond_stress(vx_scene* scene, float* ratio, float* force, uint32_t* near,
                       uint32_t cap, uint32_t* near_count);

/*
 * ---- fracture on the device ----
 *
 * FractureConfig fields read by fracture::update (src/fracture.rs:12-43; the
 * reference's defaults are 35, 0.005, 1000, 3, 0.5, 0.9).
 */
typedef struct vx_fracture_config {
    double damage_rate;
    double energy_release;
    double fatigue_cycles;
    double fatigue_exponent;
    double fatigue_threshold;
    double plastic_heat_fraction;
} vx_fracture_config;

/* Energy of a fracture stage, J, summed over bonds (fracture::Dissipation). */
typedef struct vx_dissipation {
    double plastic_heat;
    double stored_plastic;
    double surface_work;
    double damage_heat;
    double released;
} vx_dissipation;

/*
 * The fracture stage of a substep (src/solver.rs:600-665): fracture::update
 * (src/fracture.rs:210-292) on every bond of the last assembly that still has
 * a neighbour and a free owner, with the frame and undamaged stiffness of that
 * assembly, the current positions and the bond's limits. It runs the plastic
 * return map, fatigue, damage and the energy split, stores the bond state
 * (plastic strain, damage, equivalent plastic strain, plastic work, fatigue
 * state) and breaks bonds whose damage reaches 1 (neighbor = VX_EMPTY, then the
 * reverse table is rebuilt). dt is the substep. out (or NULL) receives the
 * summed dissipation (a fixed-order reduction, the same bits every run);
 * out_broken (or NULL) the number of bonds broken by this call.
 */
int32_t vx_fracture_commit(vx_scene* scene, double dt, const vx_fracture_config* config, vx_dissipation* out,
                           uint32_t* out_broken);
/*
 * rebuild_clusters (src/solver.rs:828-858) on the device: connected components
 * of the bond graph. clusters[n] (or NULL) receives each REV's cluster id,
 * numbered as the reference numbers them (in order of each component's first
 * non-kinematic REV), VX_EMPTY for kinematic REVs; out_count the cluster count.
 */
int32_t vx_scene_rebuild_clusters(vx_scene* scene, uint32_t* clusters, uint32_t* out_count);
/*
 * Bond workspace last_force (src/solver.rs:638-640): per bond, the force
 * F (K (u - plastic CELL)) (1 - damage) that the last fracture commit evaluated
 * before updating the bond, f32 N, force[9n] ((axis*n+i)*3+c). A bond the
 * commit skipped keeps its previous value (zero until its first evaluation),
 * as the reference's workspace does.
 */
int32_t vx_scene_get_last_forces(vx_scene* scene, float* force);
/* Per-bond fracture state, axis-major: plastic_strain[9n] ((axis*n+i)*3+c), damage[3n],
   equivalent_plastic_strain[3n], fatigue_damage[3n]; any may be NULL. */
int32_t vx_scene_get_bond_state(vx_scene* scene, float* plastic_strain, float* damage,
                                float* equivalent_plastic_strain, float* fatigue_damage);

/*
 * ---- contacts (collision::project, src/collision.rs:33-119; contact
 * velocities, :122-300) ----
 *
 * vx_contact_project runs the contact projection over the scene's positions,
 * with its previous positions (the substep's starts, VX_FIELD_PREVIOUS) as
 * the swept starts: candidate pairs from the swept bin boxes (:376-444)
 * without the intact-lattice pairs of each elementary cell (:505-540), then
 * up to six ordered sweeps that separate overlapping or crossing pairs
 * (:51-103). Positions and previous positions are corrected in place;
 * targeted axes (the scene's target mask) have zero inverse mass. The
 * contacts, sorted by pair with the first one of each pair kept, stay on the
 * device for vx_contact_resolve_velocities and vx_scene_get_contacts. The
 * rest positions that decide the intact-lattice pairs are the positions the
 * scene was created with.
 */
/* Previous positions of every REV, xyz[3n] (AoS): the swept starts of the
   next contact projection. A page-locked buffer is copied directly. */
int32_t vx_scene_set_previous(vx_scene* scene, const double* xyz);
typedef struct vx_contact_stats {
    uint64_t candidates;  /* pairs whose swept boxes share a bin, one REV not kinematic */
    uint64_t pairs;       /* after the intact-lattice filter */
    uint32_t contacts;
    uint32_t sweeps;
    uint32_t live_max;    /* most pairs replayed in one sweep */
    uint32_t redone;      /* sweeps replayed because a REV moved farther than its bound */
    uint32_t launches;    /* kernels launched by the call */
    uint64_t stored;      /* most pairs stored for one sweep: those that can act in it */
} vx_contact_stats;
typedef struct vx_contact_heat {
    double restitution;  /* J, kinetic loss of the normal impulses */
    double friction;     /* J, kinetic loss of the friction impulses */
} vx_contact_heat;
int32_t vx_contact_project(vx_scene* scene, vx_contact_stats* out);
/* resolve_velocities_with_precontact over the current contacts; pre_contact 0
   uses the current velocities as the pre-contact ones (resolve_velocities),
   1 the last step's drift velocities (as the step does). */
int32_t vx_contact_resolve_velocities(vx_scene* scene, int32_t pre_contact, double restitution, double friction,
                                      vx_contact_heat* out);
/* Contacts as (i, j, normal, new_impact); normal is the signed axis
   +-(axis + 1). capacity 0 only reports the count. */
int32_t vx_scene_get_contacts(vx_scene* scene, uint32_t capacity, uint32_t* i, uint32_t* j, int32_t* normal,
                              uint8_t* new_impact, uint32_t* out_count);
/* Replaces the current contacts (for velocity resolution of given contacts). */
int32_t vx_scene_set_contacts(vx_scene* scene, uint32_t count, const uint32_t* i, const uint32_t* j,
                              const int32_t* normal, const uint8_t* new_impact);

/*
 * ---- the fixed step on the device ----
 *
 * One call of solver::step_with_axis_targets_and_loads (src/solver.rs:438-700)
 * restricted to the elastic path, for every substep:
 *   - the explicit prediction (:495-517): free REVs gain gravity * h of
 *     velocity, targeted axes get zero velocity, x += v h, then targeted axes
 *     are set to their targets; the result is the predicted position;
 *   - the rotation fit, then up to corotation_iterations passes (assembly,
 *     solve, x += dx), re-fitting between passes and stopping early when the
 *     largest angle change is <= corotation_tolerance and the pass residual is
 *     <= pass.tolerance (:546-570);
 *   - the velocity update (:667-681): targeted axes (x - previous) / h, free
 *     axes drift + (x - predicted) / h.
 * Kinematic REVs do not move. The targets, loads (applied_loads: persistent
 * force + acceleration * mass + per-step loads) and masses are the scene's
 * current ones. Tools, contacts, thermal transport and the fracture commit are
 * outside this path. pass.h is ignored (h = fixed_dt / substeps).
 */
typedef struct vx_step_params {
    double fixed_dt;                 /* s (SceneConfig::fixed_dt) */
    uint32_t substeps;               /* >= 1 */
    uint32_t corotation_iterations;  /* passes per substep, >= 1 */
    double corotation_tolerance;     /* rad */
    double gravity[3];               /* m/s^2 */
    vx_pass_params pass;             /* solve of every pass; reuse_preconditioner applies from
                                        the second pass of a substep on, as the reference's CPU path */
    int32_t fracture;                /* 1: the fracture stage after the passes of every substep */
    vx_fracture_config fracture_config;
    int32_t contact;                 /* 1: contact projection and contact velocities every substep */
    double restitution;              /* FractureConfig::restitution, [0, 1] */
    double friction;                 /* FractureConfig::friction, >= 0 */
} vx_step_params;

typedef struct vx_step_stats {
    uint32_t passes;                 /* passes run, all substeps */
    uint32_t pcg_iterations;         /* PCG (inner) iterations, all passes */
    double residual;                 /* residual of the last pass (Scene::solver_residual) */
    double max_angle;                /* largest angle change of the last fit, rad */
    int32_t converged;               /* every pass reached its tolerance */
    uint32_t broken;                 /* bonds broken by the fracture stages */
    vx_dissipation dissipation;      /* summed over the fracture stages */
    uint32_t contacts;               /* contacts found, summed over substeps */
    double restitution_heat;         /* J, contact restitution loss, summed over substeps */
    double friction_heat;            /* J, contact friction loss, summed over substeps */
} vx_step_stats;

int32_t vx_scene_step(vx_scene* scene, const vx_step_params* params, vx_step_stats* out);
/* Velocities, m/s, AoS n x 3 like positions. */
int32_t vx_scene_set_velocities(vx_scene* scene, const double* xyz);
int32_t vx_scene_get_velocities(vx_scene* scene, double* xyz);
/*
 * Sets (op 0) or adds to (op 1) the velocity of count REVs: index[count],
 * value[3 * count]. Axes that are currently targeted keep zero velocity, as
 * set_velocity and apply_impulse do (src/solver.rs:207-255).
 */
int32_t vx_scene_update_velocities(vx_scene* scene, uint32_t count, const uint32_t* index,
                                   const double* value, int32_t op);
/*
 * Indexed access to one per-REV vector field (VX_FIELD_POSITION or
 * VX_FIELD_VELOCITY) of count REVs: index[count], xyz[3 * count]. Writes
 * store the given values on every axis, with no target handling; they serve
 * host calls that change a few REVs (fix_voxel_axes, apply_impulse).
 */
enum { VX_FIELD_POSITION = 0, VX_FIELD_VELOCITY = 1, VX_FIELD_PREVIOUS = 2 };
int32_t vx_scene_read_revs(vx_scene* scene, int32_t field, uint32_t count, const uint32_t* index, double* xyz);
int32_t vx_scene_write_revs(vx_scene* scene, int32_t field, uint32_t count, const uint32_t* index,
                            const double* xyz);

/*
 * ---- scene pool: many scenes resident in one arena, solved together ----
 *
 * Batched and served forms (no counterpart in the reference, which steps one
 * scene at a time). A pool reserves device memory for max_revs REVs (in
 * 256-REV tiles) and max_slots scenes up front; vx_pool_add places a scene in
 * the first free tile range that holds it and returns VX_OOM when none does
 * (admission by footprint). Scenes keep their state on the device between
 * calls. `enabled[max_slots]` selects the slots a call works on (NULL = every
 * occupied slot); the others are untouched. vx_pool_pass solves every selected
 * scene's corotational pass together in the VX_PRECISION_MIXED form with
 * per-scene scalars, so a scene's result does not depend on the other scenes
 * in the call. out[max_slots] receives per-slot statistics. Per-slot arrays
 * use the layouts of the single-scene calls for that scene's n REVs.
 */
#define VX_POOL_MATERIALS 16
typedef struct vx_pool vx_pool;
int32_t vx_pool_create(vx_ctx* ctx, uint64_t max_revs, uint32_t max_slots, vx_pool** out_pool);
int32_t vx_pool_destroy(vx_pool* pool);
uint64_t vx_pool_footprint_bytes(uint64_t max_revs, uint32_t max_slots);
uint32_t vx_pool_capacity_slots(vx_pool* pool);
int32_t vx_pool_free_revs(vx_pool* pool, uint64_t* out_free_revs, uint64_t* out_largest_range);
int32_t vx_pool_add(vx_pool* pool, const vx_scene_desc* desc, uint32_t* out_slot);
int32_t vx_pool_remove(vx_pool* pool, uint32_t slot);
int32_t vx_pool_set_positions(vx_pool* pool, uint32_t slot, const double* xyz);
int32_t vx_pool_get_positions(vx_pool* pool, uint32_t slot, double* xyz);
int32_t vx_pool_get_rotations(vx_pool* pool, uint32_t slot, double* xyzw);
int32_t vx_pool_set_targets(vx_pool* pool, uint32_t slot, const uint8_t* mask, const double* xyz);
/*
 * Moving targets: REVs whose target mask also has VX_TARGET_MOVING set get
 * their targeted axes advanced by delta[3 * slot + a] for every selected slot
 * (a prescribed-displacement tool that moves each step). delta[3 * max_slots].
 */
#define VX_TARGET_MOVING 8u
int32_t vx_pool_advance_targets(vx_pool* pool, const uint8_t* enabled, const double* delta);
int32_t vx_pool_set_loads(vx_pool* pool, uint32_t slot, const double* xyz);
int32_t vx_pool_set_predicted(vx_pool* pool, uint32_t slot, const double* xyz);
/* Velocities of one slot's REVs (zero when the scene is added). */
int32_t vx_pool_set_velocities(vx_pool* pool, uint32_t slot, const double* xyz);
int32_t vx_pool_get_velocities(vx_pool* pool, uint32_t slot, double* xyz);
int32_t vx_pool_fit_rotations(vx_pool* pool, const uint8_t* enabled, double* out_max_angle);
int32_t vx_pool_pass(vx_pool* pool, const uint8_t* enabled, const vx_pass_params* params, vx_pass_stats* out);
int32_t vx_pool_bond_stress(vx_pool* pool, uint32_t slot, float* ratio, float* force, uint32_t* near,
                            uint32_t cap, uint32_t* near_count);
/*
 * vx_scene_step for every selected slot together (params.pass.precision must
 * be VX_PRECISION_MIXED). A slot that meets the early-exit rule leaves the
 * remaining passes of its substep while the others continue; each slot's
 * result is the same whichever other slots share the call. out[max_slots].
 */
int32_t vx_pool_step(vx_pool* pool, const uint8_t* enabled, const vx_step_params* params, vx_step_stats* out);
/* Previous positions of a slot (the swept starts of the contact stage). */
int32_t vx_pool_set_previous(vx_pool* pool, uint32_t slot, const double* xyz);
int32_t vx_pool_get_previous(vx_pool* pool, uint32_t slot, double* xyz);
/* The contact projection of every selected slot, each on its own (pairs never
   join two slots); slot_contacts[max_slots] (or NULL) receives the contacts
   per slot. With contact = 1, vx_pool_step runs the contact stage for every
   slot as vx_scene_step does; its per-slot contact heat is the pool-wide total,
   like its broken-bond count. Pool keys hold at most 1024 slots. */
int32_t vx_pool_contact_project(vx_pool* pool, const uint8_t* enabled, vx_contact_stats* out,
                                uint32_t* slot_contacts);
int32_t vx_pool_checkpoint(vx_pool* pool, int32_t op);

/*
 * ---- served form: a request loop that keeps scenes resident ----
 *
 * No counterpart in the reference. A vx_server owns a host thread, a CUDA
 * stream and one pool. vx_server_submit copies a scene and queues it; at every
 * round boundary the thread admits queued scenes in arrival order while a slot
 * and a tile range of the pool are free (admission by memory footprint; the
 * pool's capacity is the HBM budget), then advances every resident scene's
 * moving targets by target_velocity * fixed_dt and runs one fixed step of all
 * resident scenes together (vx_pool_step), so requests that arrive while
 * others are stepping share the device with them (continuous batching). A
 * scene leaves after plan.steps steps; its result and final positions wait for
 * vx_server_wait. Each scene's result is the one it gets alone: pool slots
 * keep per-scene scalars. Latency of a scene-step is the time of the round it
 * stepped in.
 */
typedef struct vx_server vx_server;

typedef struct vx_server_config {
    uint64_t max_revs;            /* pool capacity in REVs; 0 = hbm_fraction of the device memory */
    double hbm_fraction;          /* budget used when max_revs == 0 (for example 0.8) */
    uint32_t max_slots;           /* resident scenes at most */
    vx_step_params step;          /* the step every scene runs (pass.precision VX_PRECISION_MIXED) */
    uint32_t lanes;               /* 0 or 1: one pool. 2..4: one pool, stream and thread per size
                                     class, so small scenes step in short rounds beside large ones */
    uint32_t lane_max_revs[3];    /* REV bound of every lane but the last (0 = 16384, 131072,
                                     1048576); the slots are split evenly, a lane but the last gets
                                     room for its slots' largest scenes (at most a quarter of the
                                     REV budget) and the last lane the rest */
} vx_server_config;

typedef struct vx_request_plan {
    uint32_t steps;               /* fixed steps to run, >= 1 */
    double target_velocity[3];    /* m/s of the targets marked VX_TARGET_MOVING (a driven tool) */
} vx_request_plan;

typedef struct vx_request_result {
    int32_t status;               /* VX_OK; VX_NOT_CONVERGED if a pass missed its tolerance; other
                                     codes when the request failed */
    uint32_t n;                   /* REVs */
    uint32_t steps_done;
    uint32_t passes;              /* corotational passes run */
    uint64_t pcg_iterations;
    double worst_residual;        /* largest pass residual over all steps */
    double queued_s;              /* submission to admission */
    double run_s;                 /* admission to completion */
} vx_request_result;

typedef struct vx_server_stats {
    uint64_t submitted, completed, failed;
    uint32_t resident, queued;
    uint64_t rounds;              /* batched steps run */
    uint64_t scene_steps;
    uint64_t solves;              /* corotational passes, each solved to its tolerance */
    double elapsed_s;             /* since creation */
    double busy_s;                /* inside batched steps */
    double p50_step_ms, p99_step_ms, max_step_ms;  /* per scene-step latency */
    uint64_t pool_revs;           /* pool capacity */
    uint64_t pool_bytes;          /* device bytes of the pool */
    double worst_residual;        /* largest pass residual of any scene-step so far */
    uint64_t not_converged;       /* scene-steps with a pass that missed its tolerance */
} vx_server_stats;

int32_t vx_server_create(vx_ctx* ctx, const vx_server_config* config, vx_server** out_server);
/* mask[n] / xyz[3n] are the scene's targets (VX_TARGET_MOVING marks moving ones), or NULL. */
int32_t vx_server_submit(vx_server* server, const vx_scene_desc* desc, const uint8_t* target_mask,
                         const double* target, const vx_request_plan* plan, uint64_t* out_ticket);
/*
 * Waits up to timeout_s for a request. Returns VX_TIMEOUT while it is still
 * queued or running; once it has finished, fills out (and positions[3n] when
 * not NULL), releases the request and returns VX_OK.
 */
int32_t vx_server_wait(vx_server* server, uint64_t ticket, double timeout_s, vx_request_result* out,
                       double* positions);
int32_t vx_server_get_stats(vx_server* server, vx_server_stats* out);
/* Stops after the current round; queued and resident requests are dropped. */
int32_t vx_server_destroy(vx_server* server);
void* vx_pool_stream(vx_pool* pool);

/* ---- state checkpoint and measurement hooks (no counterpart in the reference) ---- */

/* op 0 saves the scene's positions and rotations on the device, op 1 restores them. */
int32_t vx_scene_checkpoint(vx_scene* scene, int32_t op);
/* The scene's CUDA stream (a cudaStream_t), for callers that order or time work around it. */
void* vx_scene_stream(vx_scene* scene);
/*
 * Autotuner (no counterpart in the reference). After a pass has assembled the
 * scene, times a 64-iteration inner solve of the given precision for every
 * candidate launch configuration and keeps the fastest for the scene's later
 * passes (VX_KERNEL_AUTO follows it):
 *   - the streaming kernels with a register budget of 3, 4 or 5 blocks of 256
 *     threads per SM (candidate_blocks = that budget);
 *   - for MIXED, when the scene fits on chip, the persistent forms
 *     (candidate_blocks = VX_PERSIST_*): the brick plan with one or two
 *     threads per REV and tiles of at least 256 or 128 REVs per block, and
 *     the contiguous-range plan with the classic two reductions per
 *     iteration (at 512, 608, 768 or 896 threads per block) or with one.
 * With cache_path (or NULL), a choice found there for this GPU, precision and
 * scene size (log2 of the REV count) is applied without timing, and a new
 * choice is stored. Positions and bond state are not changed; the solver's
 * work vectors are.
 */
#define VX_PERSIST_BRICK_T1_256 1   /* brick plan, 1 thread per REV, >= 256 REVs per block */
#define VX_PERSIST_BRICK_T2_256 2   /* brick plan, 2 threads per REV, >= 256 REVs per block */
#define VX_PERSIST_BRICK_T1_128 3   /* brick plan, 1 thread per REV, >= 128 REVs per block */
#define VX_PERSIST_BRICK_T2_128 4   /* brick plan, 2 threads per REV, >= 128 REVs per block */
#define VX_PERSIST_RANGE 5          /* contiguous-range plan (classic two-reduction recurrence) */
#define VX_PERSIST_EXPANDED 6       /* contiguous-range plan, one reduction per iteration */
#define VX_PERSIST_RANGE_608 7      /* contiguous-range plan, 608 threads per block (up to 3 REVs each) */
#define VX_PERSIST_RANGE_768 8      /* contiguous-range plan, 768 threads per block (1 REV each) */
#define VX_PERSIST_RANGE_896 9      /* contiguous-range plan, 896 threads per block (up to 2 REVs each) */
typedef struct vx_tune_result {
    int32_t kernel;               /* VX_KERNEL_STREAMING or VX_KERNEL_PERSISTENT */
    int32_t blocks_per_sm;        /* streaming: register budget; persistent: VX_PERSIST_* form */
    double us_per_iteration;      /* of the chosen configuration */
    int32_t from_cache;           /* 1: read from cache_path, nothing timed */
    uint32_t candidates;          /* timed configurations (at most 12) */
    int32_t candidate_kernel[12];
    int32_t candidate_blocks[12];
    double candidate_us[12];
} vx_tune_result;
int32_t vx_scene_autotune(vx_scene* scene, int32_t precision, const char* cache_path, vx_tune_result* out);

/*
 * Device time of the inner-solve kernels on the scene's assembled system, CUDA
 * events on the scene's stream, averaged over reps launches; with flush (a
 * device buffer of flush_bytes) written before each launch so L2 starts cold.
 * out_us[5]: streaming matvec us, streaming update us, and for the MIXED
 * precision when the on-chip form fits: its us per iteration over a 64-iteration
 * solve, that solve's iterations, and its form (1 = brick plan with one grid
 * reduction per iteration, 2 = contiguous-range plan, 3 = contiguous-range plan
 * with one reduction per iteration, 0 = none).
 * The streaming kernels are timed alone, one launch of each per rep after the
 * flush (when given), on the scene's assembled system.
 */
int32_t vx_scene_kernel_times(vx_scene* scene, int32_t precision, uint32_t reps, void* flush,
                              uint64_t flush_bytes, double* out_us);

#ifdef __cplusplus
}
#endif
#endif /* VXCOROT_H */
