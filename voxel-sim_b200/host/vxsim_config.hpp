// vxsim_config.hpp — scene configuration files (RON) of Voxel-sim.
//
// SceneConfig (src/scene.rs:215-303) and FractureConfig (src/fracture.rs:10-60)
// are read from RON text with the reference's rules: every field is required
// except cuda_iterations (default 160) and cpu_preconditioner (default
// incomplete_cholesky0); unknown fields are errors; the values must pass the
// same validation, whose failure message is "Invalid scene parameters".
#pragma once

#include <array>
#include <cstdint>
#include <string>

#include "vxsim_solver.hpp"

namespace vxsim {

struct FractureSettings {
    float damage_rate = 35.0f;
    float energy_release = 0.005f;
    uint64_t propagation_delay = 1;
    float fatigue_cycles = 1000.0f;
    float fatigue_exponent = 3.0f;
    float fatigue_threshold = 0.5f;
    float plastic_heat_fraction = 0.9f;
    uint64_t fragment_min_size = 10;
    uint64_t cluster_interval = 10;
    float friction = 0.35f;
    float restitution = 0.1f;
    bool validate() const;  // FractureConfig::validate, src/fracture.rs:45-60
};

struct SceneFileConfig {
    std::array<uint64_t, 3> dimensions{1, 1, 1};
    std::array<uint64_t, 3> branch_dimensions{0, 0, 0};
    std::array<uint64_t, 3> ground_dimensions{1, 1, 1};
    std::array<uint64_t, 3> tool_dimensions{2, 2, 2};
    std::array<float, 3> fibers{0.f, 0.f, 1.f};
    float anisotropy = 0.f;
    std::array<float, 3> gravity{0.f, 0.f, -9.81f};
    float fixed_dt = 0.001f;
    uint64_t substeps = 4;
    uint64_t iterations = 80;
    uint64_t cuda_iterations = 160;
    std::string cpu_preconditioner = "incomplete_cholesky0";  // or "block_jacobi"
    float solver_relative_tolerance = 1e-5f;
    float corotation_tolerance = 1e-5f;
    uint64_t corotation_iterations = 2;
    FractureSettings fracture;
    float initial_speed = 0.f;
    std::array<float, 3> tool_start{0.f, 0.f, 0.f};

    // SceneConfig::validate (src/scene.rs:258-297): nullptr when valid.
    const char* validate() const;
    // The fields the elastic step reads, with the GPU iteration cap.
    SceneConfig solver_config() const;
};

// Parses RON text; on failure returns false with a message naming the field
// or the position of the syntax error.
bool parse_scene_config(const std::string& text, SceneFileConfig& out, std::string& error);
bool load_scene_config(const std::string& path, SceneFileConfig& out, std::string& error);

}  // namespace vxsim
