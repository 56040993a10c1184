// vxsim_solver.cpp — the solver:: mirror of vxsim_solver.hpp.
#include "vxsim_solver.hpp"

namespace vxsim {

namespace {

constexpr float kCell = 0.01f;  // CELL, src/scene.rs

}  // namespace

Scene::Scene(vx_ctx* ctx, const std::vector<VoxelSpawn>& voxels, const std::vector<vx_material>& materials,
             const SceneConfig& cfg)
    : config(cfg), n_(voxels.size()) {
    const size_t n = n_;
    std::vector<int32_t> cells(3 * n);
    std::vector<double> pos(3 * n);
    std::vector<uint32_t> mat(n), nbr(3 * n);
    std::vector<float> fib(3 * n), ani(n);
    kinematic.assign(n, 0);
    mass.assign(n, 0.f);
    external_forces.assign(n, Vec3{});
    external_accelerations.assign(n, Vec3{});
    axis_targets.assign(n, AxisTargets{});
    for (size_t i = 0; i < n; ++i) {
        const VoxelSpawn& v = voxels[i];
        if (v.material >= materials.size()) {
            status_ = VX_BAD_INPUT;
            return;
        }
        for (int a = 0; a < 3; ++a) {
            cells[3 * i + a] = v.cell[a];
            // key * CELL + CELL / 2 in f32 (src/scene.rs:1589-1592)
            pos[3 * i + a] = (double)((float)v.cell[a] * kCell + kCell * 0.5f);
            fib[3 * i + a] = v.fiber[a];
        }
        mat[i] = v.material;
        ani[i] = v.anisotropy;
        kinematic[i] = v.kinematic ? 1 : 0;
        mass[i] = materials[v.material].density * (kCell * kCell * kCell);
    }
    status_ = vx_build_topology(ctx, cells.data(), kinematic.data(), (uint32_t)n, nbr.data());
    if (status_ != VX_OK) return;
    vx_scene_desc d{};
    d.n = (uint32_t)n;
    d.position = pos.data();
    d.kinematic = kinematic.data();
    d.mass = mass.data();
    d.material = mat.data();
    d.materials = materials.data();
    d.material_count = (uint32_t)materials.size();
    d.fiber = fib.data();
    d.anisotropy = ani.data();
    d.neighbor = nbr.data();
    status_ = vx_scene_create(ctx, &d, &handle_);
    if (status_ != VX_OK) {
        handle_ = nullptr;
        return;
    }
    status_ = rebuild_clusters();  // Scene::from_voxels ends with it (src/scene.rs:571)
}

std::vector<uint32_t> Scene::neighbors() const {
    std::vector<uint32_t> out(3 * n_);
    if (handle_ && n_) vx_scene_get_neighbors(handle_, out.data());
    return out;
}

std::vector<float> Scene::bond_damage() const {
    std::vector<float> out(3 * n_);
    if (handle_ && n_) vx_scene_get_bond_state(handle_, nullptr, out.data(), nullptr, nullptr);
    return out;
}

int32_t Scene::rebuild_clusters(std::vector<uint32_t>* clusters) {
    if (!handle_) return VX_BAD_INPUT;
    if (clusters) clusters->assign(n_, 0);
    uint32_t count = 0;
    const int32_t r = vx_scene_rebuild_clusters(handle_, clusters && n_ ? clusters->data() : nullptr, &count);
    if (r == VX_OK) cluster_count = count;
    return r;
}

Scene::~Scene() {
    if (handle_) vx_scene_destroy(handle_);
}

std::vector<std::array<double, 3>> Scene::positions() const {
    std::vector<std::array<double, 3>> out(n_);
    if (handle_ && n_) vx_scene_get_positions(handle_, out[0].data());
    return out;
}
std::vector<std::array<double, 3>> Scene::velocities() const {
    std::vector<std::array<double, 3>> out(n_);
    if (handle_ && n_) vx_scene_get_velocities(handle_, out[0].data());
    return out;
}
std::array<double, 3> Scene::position(size_t i) const {
    std::array<double, 3> out{};
    const uint32_t idx = (uint32_t)i;
    if (handle_ && i < n_) vx_scene_read_revs(handle_, VX_FIELD_POSITION, 1, &idx, out.data());
    return out;
}
std::array<double, 3> Scene::velocity(size_t i) const {
    std::array<double, 3> out{};
    const uint32_t idx = (uint32_t)i;
    if (handle_ && i < n_) vx_scene_read_revs(handle_, VX_FIELD_VELOCITY, 1, &idx, out.data());
    return out;
}

namespace solver {

namespace {

Status err(const char* m) { return Status{m}; }

// A scene whose creation failed has no device state to change.
constexpr const char* kNotResident = "scene is not resident on the device";

void write_velocity(Scene& s, size_t voxel, const std::array<double, 3>& v) {
    const uint32_t idx = (uint32_t)voxel;
    vx_scene_write_revs(s.handle(), VX_FIELD_VELOCITY, 1, &idx, v.data());
}

}  // namespace

// src/solver.rs:163-175
Status set_force(Scene& s, size_t voxel, Vec3 force) {
    if (voxel >= s.size()) return err("voxel index out of range");
    if (s.kinematic[voxel]) return err("cannot apply a force to a fixed voxel");
    if (!force.is_finite()) return err("force must be finite");
    s.external_forces[voxel] = force;
    return {};
}

// src/solver.rs:177-184
Status add_force(Scene& s, size_t voxel, Vec3 force) {
    if (voxel >= s.size()) return err("voxel index out of range");
    return set_force(s, voxel, s.external_forces[voxel] + force);
}

// src/solver.rs:186-205
Status set_acceleration(Scene& s, size_t voxel, Vec3 acceleration) {
    if (voxel >= s.size()) return err("voxel index out of range");
    if (s.kinematic[voxel]) return err("cannot accelerate a fixed voxel");
    if (!acceleration.is_finite()) return err("acceleration must be finite");
    if (!(acceleration * s.mass[voxel]).is_finite()) return err("acceleration is too large for this voxel's mass");
    s.external_accelerations[voxel] = acceleration;
    return {};
}

// src/solver.rs:207-228
Status set_velocity(Scene& s, size_t voxel, Vec3 velocity) {
    if (voxel >= s.size()) return err("voxel index out of range");
    if (!s.ok()) return err(kNotResident);
    if (s.kinematic[voxel]) return err("cannot set velocity on a fixed voxel");
    if (!velocity.is_finite()) return err("velocity must be finite");
    std::array<double, 3> v{};
    for (int a = 0; a < 3; ++a) v[a] = s.axis_targets[voxel][a].has_value() ? 0.0 : (double)velocity[a];
    write_velocity(s, voxel, v);
    return {};
}

// src/solver.rs:230-255: the new velocity is formed in f32, as Vec3 arithmetic
Status apply_impulse(Scene& s, size_t voxel, Vec3 impulse) {
    if (voxel >= s.size()) return err("voxel index out of range");
    if (!s.ok()) return err(kNotResident);
    if (s.kinematic[voxel]) return err("cannot impulse a fixed voxel");
    if (!impulse.is_finite()) return err("impulse must be finite");
    const std::array<double, 3> cur = s.velocity(voxel);
    const Vec3 velocity = Vec3{(float)cur[0], (float)cur[1], (float)cur[2]} + impulse / s.mass[voxel];
    if (!velocity.is_finite()) return err("impulse would produce a non-finite velocity");
    std::array<double, 3> v{};
    for (int a = 0; a < 3; ++a) v[a] = s.axis_targets[voxel][a].has_value() ? 0.0 : (double)velocity[a];
    write_velocity(s, voxel, v);
    return {};
}

// src/solver.rs:257-265
Status clear_applied_actions(Scene& s, size_t voxel) {
    if (voxel >= s.size()) return err("voxel index out of range");
    s.external_forces[voxel] = Vec3{};
    s.external_accelerations[voxel] = Vec3{};
    return {};
}

// src/solver.rs:267-289: validated before anything changes; fixed axes move
// to their coordinates now and lose their velocity
Status fix_voxel_axes(Scene& s, size_t voxel, AxisTargets coordinates) {
    if (voxel >= s.size()) return err("voxel index out of range");
    for (const auto& c : coordinates)
        if (c.has_value() && !std::isfinite(*c)) return err("coordinates must be finite");
    if (!s.ok()) return err(kNotResident);
    s.axis_targets[voxel] = coordinates;
    std::array<double, 3> p = s.position(voxel), v = s.velocity(voxel);
    bool moved = false;
    for (int a = 0; a < 3; ++a)
        if (coordinates[a].has_value()) {
            p[a] = (double)*coordinates[a];
            v[a] = 0.0;
            moved = true;
        }
    if (moved) {
        const uint32_t idx = (uint32_t)voxel;
        vx_scene_write_revs(s.handle(), VX_FIELD_POSITION, 1, &idx, p.data());
        vx_scene_write_revs(s.handle(), VX_FIELD_VELOCITY, 1, &idx, v.data());
    }
    return {};
}

// src/solver.rs:290-293
Status fix_voxel_at(Scene& s, size_t voxel, Vec3 coordinate) {
    return fix_voxel_axes(s, voxel, AxisTargets{coordinate.x, coordinate.y, coordinate.z});
}

// src/solver.rs:294-305: fixes the chosen axes at their current (f32) coordinates
Status fix_voxel(Scene& s, size_t voxel, std::array<bool, 3> axes) {
    if (voxel >= s.size()) return err("voxel index out of range");
    if (!s.ok()) return err(kNotResident);
    const std::array<double, 3> p = s.position(voxel);
    AxisTargets t{};
    for (int a = 0; a < 3; ++a)
        if (axes[a]) t[a] = (float)p[a];
    return fix_voxel_axes(s, voxel, t);
}

// src/solver.rs:306-320
Status fix_voxel_axis(Scene& s, size_t voxel, size_t axis, std::optional<float> coordinate) {
    if (axis >= 3) return err("axis must be 0 (X), 1 (Y), or 2 (Z)");
    if (voxel >= s.size()) return err("voxel index out of range");
    AxisTargets t = s.axis_targets[voxel];
    t[axis] = coordinate;
    return fix_voxel_axes(s, voxel, t);
}

// src/solver.rs:321-323
Status release_voxel(Scene& s, size_t voxel) { return fix_voxel_axes(s, voxel, AxisTargets{}); }

int32_t step(Scene& s) { return step_with_axis_targets_and_loads(s, {}, {}); }

// src/solver.rs:422-428
int32_t step_with_targets(Scene& s, const std::vector<std::optional<Vec3>>& targets) {
    std::vector<AxisTargets> axes(targets.size());
    for (size_t i = 0; i < targets.size(); ++i)
        if (targets[i].has_value()) axes[i] = AxisTargets{targets[i]->x, targets[i]->y, targets[i]->z};
    return step_with_axis_targets_and_loads(s, axes, {});
}

int32_t step_with_axis_targets(Scene& s, const std::vector<AxisTargets>& targets) {
    return step_with_axis_targets_and_loads(s, targets, {});
}

// src/solver.rs:438-474: merged targets (explicit per-step coordinates
// override persistent ones), applied_loads, then the device step
int32_t step_with_axis_targets_and_loads(Scene& s, const std::vector<AxisTargets>& targets,
                                         const std::vector<Vec3>& loads) {
    const size_t n = s.size();
    if (!s.ok() || (!targets.empty() && targets.size() != n) || (!loads.empty() && loads.size() != n))
        return VX_BAD_INPUT;
    std::vector<uint8_t> mask(n, 0);
    std::vector<double> tgt(3 * n, 0.0), applied(3 * n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            std::optional<float> t = !targets.empty() && targets[i][a].has_value() ? targets[i][a]
                                                                                    : s.axis_targets[i][a];
            if (t.has_value()) {
                if (!std::isfinite(*t)) return VX_BAD_INPUT;
                mask[i] |= (uint8_t)(1u << a);
                tgt[3 * i + a] = (double)*t;
            }
        }
        if (!s.kinematic[i]) {
            const Vec3 extra = loads.empty() ? Vec3{} : loads[i];
            const Vec3 f = s.external_forces[i] + s.external_accelerations[i] * s.mass[i] + extra;
            for (int a = 0; a < 3; ++a) applied[3 * i + a] = (double)f[a];
        }
    }
    int32_t r = n ? vx_scene_set_targets(s.handle(), mask.data(), tgt.data()) : VX_OK;
    if (r == VX_OK && n) r = vx_scene_set_loads(s.handle(), applied.data());
    if (r != VX_OK) return r;
    vx_step_params p{};
    p.fixed_dt = s.config.fixed_dt;
    p.substeps = s.config.substeps;
    p.corotation_iterations = s.config.corotation_iterations;
    p.corotation_tolerance = s.config.corotation_tolerance;
    for (int a = 0; a < 3; ++a) p.gravity[a] = s.config.gravity[a];
    p.pass.h = (double)s.config.fixed_dt / (double)s.config.substeps;
    p.pass.tolerance = s.config.solver_relative_tolerance;
    p.pass.max_iterations = s.config.iterations;
    p.pass.precision = s.config.precision;
    p.pass.reuse_preconditioner = s.config.reuse_preconditioner ? 1 : 0;
    p.pass.kernel = s.config.kernel;
    p.fracture = s.config.fracture ? 1 : 0;
    p.fracture_config = s.config.fracture_config;
    p.contact = s.config.contact ? 1 : 0;
    p.restitution = s.config.restitution;
    p.friction = s.config.friction;
    r = vx_scene_step(s.handle(), &p, &s.last_step);
    if (r != VX_OK && r != VX_NOT_CONVERGED) return r;
    s.solver_residual = s.last_step.residual;
    s.broken += s.last_step.broken;
    if (s.last_step.broken > 0) {
        const int32_t rc = s.rebuild_clusters();
        if (rc != VX_OK) return rc;
    }
    return r;
}

}  // namespace solver
}  // namespace vxsim
