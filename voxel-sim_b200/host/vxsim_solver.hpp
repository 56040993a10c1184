// vxsim_solver.hpp — C++ host mirror of Voxel-sim's solver:: public API
// (src/solver.rs:163-323 and :419-445) above the C ABI of include/vxcorot.h.
//
// It stands where the reference's Rust host loop stands: the persistent
// inputs (forces, accelerations, axis targets) live on the host, as they do
// on Scene (src/scene.rs:309-351); positions, rotations, velocities and bonds
// live on the device in a vx_scene. Every function keeps the reference's
// name, argument meaning and error messages; a step merges per-step targets
// with the persistent ones, forms applied_loads = force + acceleration * mass
// + per-step loads (src/solver.rs:446-474) and runs vx_scene_step.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <optional>
#include <vector>

#include "../../include/vxcorot.h"

namespace vxsim {

// glam::Vec3 at the API (f32 components).
struct Vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    constexpr Vec3() = default;
    constexpr Vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
    static constexpr Vec3 splat(float v) { return {v, v, v}; }
    float operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
    float& operator[](int a) { return a == 0 ? x : (a == 1 ? y : z); }
    bool is_finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
    Vec3 operator+(Vec3 o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator*(float s) const { return {x * s, y * s, z * s}; }
    Vec3 operator/(float s) const { return {x / s, y / s, z / s}; }
};

// Result<(), &'static str>: no error on success, else the reference's message.
struct Status {
    const char* error = nullptr;
    bool is_ok() const { return error == nullptr; }
    bool is_err() const { return error != nullptr; }
};

using AxisTargets = std::array<std::optional<float>, 3>;

// The SceneConfig fields the elastic step reads (src/scene.rs:215-265), with
// the reference's defaults, plus the precision form and inner kernel choice.
struct SceneConfig {
    std::array<float, 3> gravity{0.f, 0.f, -9.81f};
    float fixed_dt = 0.001f;
    uint32_t substeps = 4;
    uint32_t iterations = 80;  // PCG iteration cap per pass
    float solver_relative_tolerance = 1e-5f;
    float corotation_tolerance = 1e-5f;
    uint32_t corotation_iterations = 2;
    int32_t precision = VX_PRECISION_FP64;
    int32_t kernel = VX_KERNEL_AUTO;
    bool reuse_preconditioner = true;  // the CPU path's stale factor from the second pass on
    // fracture::update after the passes of every substep (src/solver.rs:624-663),
    // with FractureConfig::default (src/fracture.rs:27-42) in its f32 values
    bool fracture = true;
    vx_fracture_config fracture_config{35.0, (double)0.005f, 1000.0, 3.0, 0.5, (double)0.9f};
    // collision::project and the contact velocities (src/solver.rs:575-690)
    bool contact = true;
    float restitution = 0.1f;  // FractureConfig::restitution
    float friction = 0.35f;    // FractureConfig::friction
};

// One REV of a lattice built from cells (Scene::from_voxels, src/scene.rs:445-573).
struct VoxelSpawn {
    std::array<int32_t, 3> cell{};
    uint32_t material = 0;
    bool kinematic = false;
    Vec3 fiber{0.f, 0.f, 1.f};  // Microstructure::fibers()
    float anisotropy = 0.f;  // VoxelSpawn::new (src/scene.rs:97-109)
};

class Scene {
public:
    // A resident scene: positions at cell centres ((cell + 1/2) * CELL), mass
    // = density * CELL^3, identity rotations, bonds between face neighbours
    // with equal kinematic flags (built on the device).
    Scene(vx_ctx* ctx, const std::vector<VoxelSpawn>& voxels, const std::vector<vx_material>& materials,
          const SceneConfig& config);
    ~Scene();
    Scene(const Scene&) = delete;
    Scene& operator=(const Scene&) = delete;

    bool ok() const { return handle_ != nullptr; }
    int32_t status() const { return status_; }
    size_t size() const { return n_; }
    vx_scene* handle() const { return handle_; }

    // device state, f64 (AoS)
    std::vector<std::array<double, 3>> positions() const;
    std::vector<std::array<double, 3>> velocities() const;
    std::array<double, 3> position(size_t i) const;
    std::array<double, 3> velocity(size_t i) const;
    // bond state, axis-major (axis * n + i): Bond::neighbor and Bond::damage
    std::vector<uint32_t> neighbors() const;
    std::vector<float> bond_damage() const;
    // rebuild_clusters (src/solver.rs:828-858): sets cluster_count; the REVs'
    // cluster ids when asked for
    int32_t rebuild_clusters(std::vector<uint32_t>* clusters = nullptr);

    SceneConfig config;
    std::vector<Vec3> external_forces;
    std::vector<Vec3> external_accelerations;
    std::vector<AxisTargets> axis_targets;
    std::vector<float> mass;
    std::vector<uint8_t> kinematic;
    vx_step_stats last_step{};
    uint64_t broken = 0;         // Scene::broken: bonds broken since creation
    size_t cluster_count = 0;    // Scene::cluster_count
    double solver_residual = 0;  // Scene::solver_residual of the last pass

private:
    vx_scene* handle_ = nullptr;
    int32_t status_ = VX_OK;
    size_t n_ = 0;
};

namespace solver {

Status set_force(Scene& scene, size_t voxel, Vec3 force);
Status add_force(Scene& scene, size_t voxel, Vec3 force);
Status set_acceleration(Scene& scene, size_t voxel, Vec3 acceleration);
Status set_velocity(Scene& scene, size_t voxel, Vec3 velocity);
Status apply_impulse(Scene& scene, size_t voxel, Vec3 impulse);
Status clear_applied_actions(Scene& scene, size_t voxel);
Status fix_voxel_axes(Scene& scene, size_t voxel, AxisTargets coordinates);
Status fix_voxel_at(Scene& scene, size_t voxel, Vec3 coordinate);
Status fix_voxel(Scene& scene, size_t voxel, std::array<bool, 3> axes);
Status fix_voxel_axis(Scene& scene, size_t voxel, size_t axis, std::optional<float> coordinate);
Status release_voxel(Scene& scene, size_t voxel);

// The step functions return the vx status of the device step (VX_OK,
// VX_NOT_CONVERGED, ...); VX_BAD_INPUT where the reference asserts (target or
// load slices of the wrong length, non-finite merged targets). A step that
// broke bonds rebuilds the clusters (src/solver.rs:741-743).
int32_t step(Scene& scene);
int32_t step_with_targets(Scene& scene, const std::vector<std::optional<Vec3>>& targets);
int32_t step_with_axis_targets(Scene& scene, const std::vector<AxisTargets>& targets);
int32_t step_with_axis_targets_and_loads(Scene& scene, const std::vector<AxisTargets>& targets,
                                         const std::vector<Vec3>& loads);

}  // namespace solver
}  // namespace vxsim
