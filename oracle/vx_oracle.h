/*
 * vx_oracle.h — CPU restatement of the Voxel-sim corotational elastic solve.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle for the CUDA path: the
 * tests, the package smoke check and the bench's CPU-baseline arm call it as
 * the checker or the timed CPU reference. The product path never links or
 * calls it.
 *
 * Every function restates the reference's algorithm (TheLastie/Voxel-sim,
 * Rust, f32 glam maths) in double precision and cites the reference lines it
 * follows. The reference itself cannot be built here (no cargo/rustc and no
 * vendored crates), so the oracle is pinned by the reference's own unit tests,
 * fixtures and kernel probes (tests/test_oracle_golden.py), which fix the
 * results to the tolerances those tests state (1e-6..2e-5 and exact ratios).
 * Bit-level parity with glam's f32 arithmetic is not pinned.
 *
 * Two PCG restatements in f32 reproduce the reference's own precision:
 *   vxo_pcg_rows_f32       — the CPU block-Jacobi loop (src/solver.rs:1833-1911)
 *   vxo_cuda_pcg_emulate   — the CUDA/PTX sequence (src/cuda_solver.rs:366-478,
 *                            src/cuda/pcg.ptx)
 */
#ifndef VX_ORACLE_H
#define VX_ORACLE_H

#include <stdint.h>
#include "../include/vxcorot.h"

#ifdef __cplusplus
extern "C" {
#endif

/* CELL and AREA are f32 constants in the reference (src/scene.rs:10-11). */
extern const double VXO_CELL;
extern const double VXO_AREA;

typedef struct vxo_scene {
    uint32_t n;
    double* pos;               /* 3n */
    double* rot;               /* 4n xyzw */
    const uint8_t* kinematic;  /* n */
    const double* mass;        /* n */
    const uint32_t* material;  /* n */
    const vx_material* materials;
    const double* fiber;       /* 3n body-frame fibre axis */
    const double* anisotropy;  /* n */
    const double* solid;       /* n */
    const double* thermal_scale; /* n */
    const double* thermal_delta; /* n */
    uint32_t* nbr;             /* 3n axis-major */
    double* formation;         /* 9n */
    double* plastic;           /* 9n */
    double* damage;            /* 3n */
    double* eq_plastic;        /* 3n Bond::equivalent_plastic_strain, or NULL (0) */
} vxo_scene;

/* Assembled system of one corotational pass (src/solver.rs:1576-1672). */
typedef struct vxo_system {
    uint32_t n;
    double* free;        /* 3n 0/1 */
    double* diag;        /* 9n projected diagonal blocks, row-major */
    double* rhs;         /* 3n projected rhs */
    double* k;           /* 27n world K of bond axis*n+i (row-major), 0 if not assembled */
    double* material_k;  /* 27n undamaged local K */
    double* frame;       /* 27n frame (row-major: frame[r*3+c], columns are the axes) */
    double* rest;        /* 9n world rest vector */
    uint8_t* state;      /* 3n: 0 = not a constraint, 1 = fracture only, 2 = assembled */
    /* constraint list in the reference's push order (axis-major, i ascending) */
    uint32_t* c_i;       /* up to 3n */
    uint32_t* c_j;
    uint32_t* c_axis;
    uint32_t c_count;
    /* incidence of assembled constraints, reference insertion order */
    uint32_t* incidence; /* 6n bond indices axis*n+i */
    uint8_t* incidence_len; /* n */
    uint32_t* partner;   /* 3n: partner j of each constraint bond at assembly time */
} vxo_system;

typedef struct vxo_limits {
    double tension, compression, shear, yield_stress, hardening, plastic_failure, ductility,
        fracture_energy;
} vxo_limits;

typedef struct vxo_fracture_config {
    double damage_rate, energy_release, fatigue_cycles, fatigue_exponent, fatigue_threshold,
        plastic_heat_fraction;
} vxo_fracture_config;

typedef struct vxo_bond {
    uint32_t neighbor;
    double formation[3];
    double plastic[3];
    double damage, equivalent_plastic_strain, plastic_work, fatigue_damage,
        previous_stress_ratio, reversal_stress_ratio, loading_increment;
} vxo_bond;

typedef struct vxo_dissipation {
    double plastic_heat, stored_plastic, surface_work, damage_heat, released;
} vxo_dissipation;

/* ---- geometry / rotation ------------------------------------------------ */
void vxo_basis(int axis, const double q[4], double frame[9]);
void vxo_slerp_half(const double a[4], const double b[4], double out[4]);
void vxo_quat_from_mat3(const double m[9], double q[4]);
double vxo_fit_rotations(vxo_scene* s);
uint32_t vxo_build_topology(const int32_t* cells, const uint8_t* kinematic, uint32_t n,
                            uint32_t* nbr);

/* ---- constitutive ------------------------------------------------------- */
int vxo_tensor_compliance(const vxo_scene* s, uint32_t n, const double frame[9], double c[9]);
void vxo_stiffness_matrix(const vxo_scene* s, uint32_t i, uint32_t j, const double frame[9],
                          double k[9]);
void vxo_bond_thermal_rest(const vxo_scene* s, uint32_t i, uint32_t j, const double frame[9],
                           double rest[3]);
void vxo_make_constraint(const vxo_scene* s, uint32_t i, int axis, uint32_t j, double frame[9],
                         double material_k[9], double k[9], double rest[3]);
void vxo_pair_limits(const vx_material* a, const vx_material* b, const double alignment[2],
                     const double anisotropy[2], vxo_limits* out);
void vxo_bond_limits(const vxo_scene* s, uint32_t i, uint32_t j, const double direction[3],
                     vxo_limits* out);
void vxo_fracture_update(vxo_bond* b, const double u_total[3], const double k[9],
                         const vxo_limits* l, double dt, const vxo_fracture_config* c,
                         vxo_dissipation* out);
void vxo_fatigue(vxo_bond* b, double signed_ratio, const vxo_fracture_config* c);
double vxo_stress_ratio(const double u_total[3], const double plastic[3], const double k[9],
                        const vxo_limits* l, double eq_plastic);

/* ---- system and solve --------------------------------------------------- */
int vxo_system_alloc(vxo_system* sys, uint32_t n);
void vxo_system_free(vxo_system* sys);
void vxo_assemble(const vxo_scene* s, const uint8_t* target_mask, const double* loads,
                  const double* predicted, double h, vxo_system* sys);
void vxo_matvec(const vxo_system* sys, const double* p, double* out);
void vxo_factor_block_jacobi(const vxo_system* sys, double* factor);
int vxo_pcg(const vxo_system* sys, const double* factor, uint32_t max_iterations,
            double tolerance, int fixed_iterations, double* dx, uint32_t* iterations,
            double* residual);
int vxo_solve_coupled(vxo_scene* s, const uint8_t* target_mask, const double* loads,
                      const double* predicted, double h, uint32_t max_iterations,
                      double tolerance, int reuse_preconditioner, double* factor,
                      vxo_system* sys, uint32_t* iterations, double* residual);
double vxo_true_residual(const vxo_system* sys, const double* dx);
void vxo_bond_stress(const vxo_scene* s, const vxo_system* sys, double* ratio, double* force);

/* ---- packed active-row system and the reference's f32 PCG loops ---------- */
uint32_t vxo_pack_rows(const vxo_system* sys, uint32_t* active, float* rhs, uint32_t* nbr6,
                       float* diag9, float* blocks54, float* inv9);
int vxo_pcg_rows_f32(uint32_t n, const float* rhs, const uint32_t* nbr6, const float* diag9,
                     const float* blocks54, uint32_t max_iterations, float tolerance,
                     int threads, float* dx, uint32_t* iterations, float* residual);
int vxo_cuda_pcg_emulate(uint32_t n, const float* rhs, const uint32_t* nbr6,
                         const float* diag9, const float* blocks54, const float* inv9,
                         uint32_t max_iterations, float tolerance, float* dx,
                         uint32_t* iterations, float* residual);

/* ---- one fixed step (src/solver.rs:440-763 without tool/thermal) --------- */
typedef struct vxo_step_config {
    double fixed_dt;
    uint32_t substeps;
    uint32_t iterations;
    double solver_tolerance;
    double corotation_tolerance;
    uint32_t corotation_iterations;
    double gravity[3];
    vxo_fracture_config fracture;
    int fracture_enabled;
    int contact_enabled;   /* collision::project and resolve_velocities_with_precontact */
    double restitution;    /* FractureConfig::restitution */
    double friction;       /* FractureConfig::friction */
} vxo_step_config;

typedef struct vxo_dynamics {
    double* velocity;        /* 3n */
    double* previous;        /* 3n */
    uint8_t* target_mask;    /* n, merged targets of this step */
    double* target;          /* 3n */
    double* applied_loads;   /* 3n */
    vxo_bond* bonds;         /* 3n fracture state (neighbor mirrored into scene->nbr) */
    double* last_force;      /* 9n */
    double solver_residual;
    uint64_t broken;
    uint64_t pcg_iterations;
    double external_work;
    double plastic_heat, stored_plastic, surface_work, damage_heat, pending_release;
    const double* rest;      /* 3n Scene::rest_positions (contacts only) */
    uint64_t contacts;       /* contacts found, summed over substeps */
    double restitution_heat, friction_heat;
} vxo_dynamics;

int vxo_step(vxo_scene* s, const vxo_step_config* cfg, vxo_dynamics* d);

/* ---- contacts (src/collision.rs) ------------------------------------------ */
/* normal: signed axis code +-(axis + 1); order: position in the push order */
typedef struct vxo_contact {
    uint32_t i, j;
    int32_t normal;
    int32_t new_impact;
    uint32_t order;
} vxo_contact;

typedef struct vxo_contact_stats {
    uint64_t candidates; /* pairs from the bins */
    uint64_t pairs;      /* after the local-continuum filter */
    uint64_t contacts;
    uint32_t sweeps;
} vxo_contact_stats;

/* bin_bounds of REV i's swept box (src/collision.rs:437-444), cell units */
void vxo_contact_box(const double* start, const double* pos, uint32_t i, int32_t lo[3], int32_t hi[3]);
/* local_continuum_pair (src/collision.rs:505-540); adj[6n] as adjacency() builds it */
int vxo_local_continuum_pair(const double* rest, const uint32_t* adj, uint32_t i, uint32_t j);
/* collision::project (src/collision.rs:33-119): positions and previous (3n) are
   corrected in place; starts are previous on entry. *out (malloc'd, caller
   frees) receives the contacts sorted by (i, j), the first of each pair kept.
   tmask (or NULL): targeted axes have zero inverse mass. */
uint32_t vxo_contact_project(uint32_t n, double* pos, double* prev, const double* rest, const uint8_t* kinematic,
                             const double* mass, const uint8_t* tmask, const uint32_t* nbr, vxo_contact** out,
                             vxo_contact_stats* st);
/* resolve_velocities_with_precontact (src/collision.rs:133-300); heat totals
   are added to *restitution_heat and *friction_heat. */
void vxo_resolve_velocities(uint32_t n, double* velocity, const double* pre_contact, const uint8_t* kinematic,
                            const double* mass, const uint8_t* tmask, const vxo_contact* contacts, uint32_t count,
                            double restitution, double friction, double* restitution_heat, double* friction_heat);

/* rebuild_clusters (src/solver.rs:828-858): union-find over every bond with a
   neighbour; non-kinematic REVs get ids in the order their components first
   appear by REV index, kinematic REVs VX_EMPTY. Returns cluster_count. */
uint32_t vxo_rebuild_clusters(uint32_t n, const uint32_t* neighbor, const uint8_t* kinematic, uint32_t* clusters);

#ifdef __cplusplus
}
#endif
#endif
