// The reference's own tests of the solver:: public API (src/solver.rs:905-1006,
// tests/supports.rs:42-54), restated against the C++ host mirror, which runs
// the step on the device. Parts that need contacts, a floor or energy
// accounting (outside the elastic path) are left out. Prints PASS/FAIL per
// test; exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "vxsim_solver.hpp"

using namespace vxsim;

static int g_failures = 0;

// The reference's Result is Err(message): compare the message, tolerating Ok.
static bool err_is(const Status& st, const char* message) {
    return st.error != nullptr && std::strcmp(st.error, message) == 0;
}
static bool g_ok = true;

#define CHECK(cond)                                                       \
    do {                                                                  \
        if (!(cond)) {                                                    \
            std::printf("  check failed at line %d: %s\n", __LINE__, #cond); \
            g_ok = false;                                                 \
        }                                                                 \
    } while (0)

// Material::table row 1 ("wood", src/material.rs:96-116 with the row
// overrides of :274-320)
static vx_material wood() {
    vx_material m{};
    m.density = 650.f;
    m.young = 10e9f;
    m.young_perp = 0.6e9f;
    m.shear = 0.65e9f;
    m.tensile_strength = 100e6f;
    m.tensile_strength_perp = 2.5e6f;
    m.compressive_strength = 50e6f;
    m.compressive_strength_perp = 2e6f;
    m.shear_strength = 12e6f;
    m.shear_strength_perp = 3e6f;
    m.yield_strength = 25e6f;
    m.hardening_modulus = 2e9f;
    m.failure_plastic_strain = 0.04f;
    m.fracture_energy = 350.f;
    m.fracture_energy_perp = 80.f;
    m.thermal_expansion_parallel = 3e-6f;
    m.thermal_expansion_perpendicular = 30e-6f;
    m.fracture_mode = VX_MIXED;
    return m;
}

static std::vector<VoxelSpawn> box(int nx, int ny, int nz, int z0, bool kinematic) {
    std::vector<VoxelSpawn> v;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                VoxelSpawn s;
                s.cell = {x, y, z0 + z};
                s.kinematic = kinematic;
                v.push_back(s);
            }
    return v;
}

// free_voxel() of src/solver.rs:893-904: one wood REV, no gravity, dt 0.01,
// one substep, one PCG iteration, one corotational pass
static SceneConfig free_voxel_config() {
    SceneConfig c;
    c.gravity = {0.f, 0.f, 0.f};
    c.fixed_dt = 0.01f;
    c.substeps = 1;
    c.iterations = 1;
    c.corotation_iterations = 1;
    return c;
}

// A step that reports its status and, on failure, the library's message.
static bool step_ok(Scene& s) {
    const int32_t st = solver::step(s);
    if (st != VX_OK) std::printf("  step status %d: %s\n", st, vx_last_error());
    return st == VX_OK;
}

static void persistent_force_and_acceleration_use_voxel_mass(vx_ctx* ctx) {
    Scene s(ctx, box(1, 1, 1, 0, false), {wood()}, free_voxel_config());
    CHECK(s.ok());
    const float mass = s.mass[0];
    CHECK(solver::set_force(s, 0, Vec3(1, 0, 0) * (3.f * mass)).is_ok());
    CHECK(solver::set_acceleration(s, 0, Vec3(0, 1, 0) * 2.f).is_ok());
    CHECK(step_ok(s));
    auto v = s.velocity(0);
    CHECK(std::fabs(v[0] - 0.03) < 1e-5);
    CHECK(std::fabs(v[1] - 0.02) < 1e-5);
    CHECK(step_ok(s));
    v = s.velocity(0);
    CHECK(std::fabs(v[0] - 0.06) < 1e-5);
    CHECK(std::fabs(v[1] - 0.04) < 1e-5);
    CHECK(solver::clear_applied_actions(s, 0).is_ok());
    CHECK(step_ok(s));
    v = s.velocity(0);
    CHECK(std::fabs(v[0] - 0.06) < 1e-5);
    CHECK(std::fabs(v[1] - 0.04) < 1e-5);
}

static void velocity_and_impulse_are_mass_consistent(vx_ctx* ctx) {
    Scene s(ctx, box(1, 1, 1, 0, false), {wood()}, free_voxel_config());
    CHECK(s.ok());
    const float mass = s.mass[0];
    CHECK(solver::set_velocity(s, 0, Vec3(1, 0, 0) * 1.5f).is_ok());
    CHECK(solver::apply_impulse(s, 0, Vec3(0, 1, 0) * (mass * 2.f)).is_ok());
    const auto v = s.velocity(0);
    CHECK(std::fabs(v[0] - 1.5) < 1e-6);
    CHECK(std::fabs(v[1] - 2.0) < 1e-6);
}

// scene() of src/solver.rs:885-892: a 2x2x2 wood block on a fixed 2x2x1 ground
static void external_actions_reject_fixed_and_missing_voxels(vx_ctx* ctx) {
    std::vector<VoxelSpawn> v = box(2, 2, 1, 0, true);
    const std::vector<VoxelSpawn> block = box(2, 2, 2, 1, false);
    v.insert(v.end(), block.begin(), block.end());
    SceneConfig c;
    c.gravity = {0.f, 0.f, 0.f};
    Scene s(ctx, v, {wood()}, c);
    CHECK(s.ok());
    size_t fixed = 0;
    while (fixed < s.size() && !s.kinematic[fixed]) ++fixed;
    const size_t free_rev = s.size() - 1;
    CHECK(err_is(solver::set_force(s, fixed, Vec3(1, 0, 0)), "cannot apply a force to a fixed voxel"));
    CHECK(err_is(solver::set_acceleration(s, fixed, Vec3(1, 0, 0)), "cannot accelerate a fixed voxel"));
    CHECK(err_is(solver::apply_impulse(s, fixed, Vec3(1, 0, 0)), "cannot impulse a fixed voxel"));
    CHECK(err_is(solver::set_velocity(s, (size_t)-1, Vec3(1, 0, 0)), "voxel index out of range"));
    CHECK(err_is(solver::set_force(s, free_rev, Vec3::splat(NAN)), "force must be finite"));
    CHECK(solver::set_force(s, free_rev, Vec3(1, 0, 0)).is_ok());
}

// tests/supports.rs:42-54 on one free REV (dt 1 ms, two substeps)
static void constraint_inputs_are_atomic_and_impulses_respect_fixed_axes(vx_ctx* ctx) {
    SceneConfig c;
    c.fixed_dt = 0.001f;
    c.substeps = 2;
    Scene s(ctx, box(1, 1, 1, 0, false), {wood()}, c);
    CHECK(s.ok());
    CHECK(solver::fix_voxel(s, 0, {true, false, true}).is_ok());
    const AxisTargets old = s.axis_targets[0];
    CHECK(solver::fix_voxel_axes(s, 0, AxisTargets{1.f, NAN, std::nullopt}).is_err());
    CHECK(s.axis_targets[0] == old);
    CHECK(err_is(solver::fix_voxel_axis(s, 0, 3, std::nullopt), "axis must be 0 (X), 1 (Y), or 2 (Z)"));
    CHECK(solver::fix_voxel(s, 100, {true, true, true}).is_err());
    const float mass = s.mass[0];
    CHECK(solver::apply_impulse(s, 0, Vec3::splat(1.f) * mass).is_ok());
    const auto v = s.velocity(0);
    CHECK(v[0] == 0.0 && v[1] == 1.0 && v[2] == 0.0);
}

// A 6x2x2 wood bar, x = 0 end fixed, the far end pulled 0.1 mm along +x by
// per-step axis targets: the targeted REVs sit on their targets and the
// interior follows monotonically along the bar.
static void axis_targets_pull_a_bar(vx_ctx* ctx) {
    std::vector<VoxelSpawn> v = box(6, 2, 2, 0, false);
    SceneConfig c;
    c.gravity = {0.f, 0.f, 0.f};
    c.substeps = 1;
    c.iterations = 2000;
    c.solver_relative_tolerance = 1e-9f;
    Scene s(ctx, v, {wood()}, c);
    CHECK(s.ok());
    for (size_t i = 0; i < s.size(); ++i)
        if (v[i].cell[0] == 0) CHECK(solver::fix_voxel(s, i, {true, true, true}).is_ok());
    const auto x0 = s.positions();
    std::vector<AxisTargets> targets(s.size());
    for (size_t i = 0; i < s.size(); ++i)
        if (v[i].cell[0] == 5) targets[i] = AxisTargets{(float)(x0[i][0] + 1e-4), (float)x0[i][1], (float)x0[i][2]};
    CHECK(solver::step_with_axis_targets(s, targets) == VX_OK);
    const auto x = s.positions();
    double ux[6] = {0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < s.size(); ++i) {
        ux[v[i].cell[0]] += (x[i][0] - x0[i][0]) / 4.0;
        if (v[i].cell[0] == 5) CHECK(x[i][0] == (double)*targets[i][0]);
        if (v[i].cell[0] == 0) CHECK(x[i][0] == x0[i][0]);
    }
    for (int k = 1; k < 6; ++k) CHECK(ux[k] > ux[k - 1]);
    CHECK(s.last_step.passes >= 1 && s.last_step.converged == 1);
    CHECK(solver::step_with_axis_targets(s, std::vector<AxisTargets>(3)) == VX_BAD_INPUT);
}

int main() {
    std::setvbuf(stdout, nullptr, _IONBF, 0);
    vx_ctx* ctx = nullptr;
    if (vx_ctx_create(0, &ctx) != VX_OK) {
        std::printf("FAIL no device: %s\n", vx_last_error());
        return 2;
    }
    struct Case {
        const char* name;
        void (*fn)(vx_ctx*);
    } cases[] = {
        {"persistent_force_and_acceleration_use_voxel_mass", persistent_force_and_acceleration_use_voxel_mass},
        {"velocity_and_impulse_are_mass_consistent", velocity_and_impulse_are_mass_consistent},
        {"external_actions_reject_fixed_and_missing_voxels", external_actions_reject_fixed_and_missing_voxels},
        {"constraint_inputs_are_atomic_and_impulses_respect_fixed_axes",
         constraint_inputs_are_atomic_and_impulses_respect_fixed_axes},
        {"axis_targets_pull_a_bar", axis_targets_pull_a_bar},
    };
    for (const Case& c : cases) {
        g_ok = true;
        std::printf("RUN  %s\n", c.name);
        c.fn(ctx);
        if (!g_ok) std::printf("  last library message: %s\n", vx_last_error());
        std::printf("%s %s\n", g_ok ? "PASS" : "FAIL", c.name);
        if (!g_ok) ++g_failures;
    }
    vx_ctx_destroy(ctx);
    return g_failures == 0 ? 0 : 1;
}
