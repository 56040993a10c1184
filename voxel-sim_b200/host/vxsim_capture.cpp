// vxsim_capture.cpp — the solver scale capture (src/bin/solver_scale_capture.rs)
// on the device step.
//
//   vxsim_capture [path] [steps] [saved_frames] [scene.ron]
//
// A 36 x 32 x 32 iron block at 293.15 K with its bottom layer fixed
// (kinematic) is stepped under gravity with no scripted motion; the CSV
// records the outer surface at saved_frames evenly spaced states:
//   H,<dt>,<steps>,<saved_frames>
//   F,<frame>,0,0,0,0,0,0,1,0,0,<broken>,<cluster_count>,0
//   V,<frame>,<sample_id>,<x>,<y>,<z>,<max bond damage>,<lost bonds>,<index>
// for every boundary REV whose index is not a multiple of 3, numbers in the
// shortest decimal form that reads back to the same f32 (Rust's `{}`). The
// scene settings are SceneConfig::default with dimensions 36 x 32 x 32 and
// fixed_dt 1 ms, or those of a RON scene file given as the fourth argument.
// The block and the fixed layer are not bonded (their kinematic flags
// differ): the block stands on the layer through the contact stage of the
// step (collision::project and the contact velocities). VXSIM_PRECISION=1
// selects the mixed-precision solve.
#include <charconv>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "vxsim_config.hpp"
#include "vxsim_materials.hpp"
#include "vxsim_solver.hpp"

using namespace vxsim;

namespace {

constexpr size_t NX = 36, NY = 32, NZ = 32;

// Rust's Display for f32: the shortest round-trip digits, never an exponent.
std::string f32_display(float v) {
    char buf[64];
    if (v != v) return "NaN";
    if (v == __builtin_inff()) return "inf";
    if (v == -__builtin_inff()) return "-inf";
    const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::fixed);
    return std::string(buf, r.ptr);
}

// (max damage over the REV's existing bonds, bonds lost) — surface_state
// (src/bin/solver_scale_capture.rs:20-46)
void surface_state(const std::vector<uint32_t>& nbr, const std::vector<float>& damage, size_t n, size_t x, size_t y,
                   size_t z, float& max_damage, unsigned& lost) {
    const size_t index = (z * NY + y) * NX + x;
    const size_t strides[3] = {1, NX, NX * NY};
    const size_t coords[3] = {x, y, z};
    const size_t extents[3] = {NX, NY, NZ};
    max_damage = 0.f;
    lost = 0;
    auto visit = [&](size_t axis, size_t owner) {
        const size_t e = axis * n + owner;
        if (nbr[e] == VX_EMPTY)
            ++lost;
        else
            max_damage = std::max(max_damage, damage[e]);
    };
    for (size_t axis = 0; axis < 3; ++axis) {
        if (coords[axis] + 1 < extents[axis]) visit(axis, index);
        if (coords[axis] > 0) visit(axis, index - strides[axis]);
    }
}

bool parse_count(const char* s, size_t& out) {
    char* end = nullptr;
    const unsigned long long v = std::strtoull(s, &end, 10);
    if (end == s || *end != '\0' || s[0] == '-') return false;
    out = (size_t)v;
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    const std::string path = argc > 1 ? argv[1] : "solver-scale-36k.csv";
    size_t steps = 176, saved_frames = 0;
    if (argc > 2 && !parse_count(argv[2], steps)) {
        std::fprintf(stderr, "invalid steps `%s`\n", argv[2]);
        return 1;
    }
    saved_frames = steps + 1;
    if (argc > 3 && !parse_count(argv[3], saved_frames)) {
        std::fprintf(stderr, "invalid saved_frames `%s`\n", argv[3]);
        return 1;
    }
    if (steps == 0 || saved_frames < 2 || saved_frames > steps + 1) {
        std::fprintf(stderr, "steps must be positive and saved_frames must be in 2..=steps+1\n");
        return 1;
    }
    SceneFileConfig file;
    file.dimensions = {NX, NY, NZ};
    file.fixed_dt = 0.001f;
    if (argc > 4) {
        std::string why;
        if (!load_scene_config(argv[4], file, why)) {
            std::fprintf(stderr, "%s: %s\n", argv[4], why.c_str());
            return 1;
        }
    }
    SceneConfig config = file.solver_config();
    if (const char* p = std::getenv("VXSIM_PRECISION")) config.precision = std::atoi(p);

    const int iron = material_component_id("iron");
    std::vector<VoxelSpawn> spawns;
    spawns.reserve(NX * NY * NZ);
    for (size_t z = 0; z < NZ; ++z)
        for (size_t y = 0; y < NY; ++y)
            for (size_t x = 0; x < NX; ++x) {
                VoxelSpawn v;
                v.cell = {(int32_t)x, (int32_t)y, (int32_t)z};
                v.material = (uint32_t)iron;
                v.kinematic = z == 0;
                v.anisotropy = 0.f;
                spawns.push_back(v);
            }
    vx_ctx* ctx = nullptr;
    if (vx_ctx_create(0, &ctx) != VX_OK) {
        std::fprintf(stderr, "no device: %s\n", vx_last_error());
        return 1;
    }
    int rc = 0;
    {
        Scene scene(ctx, spawns, builtin_materials(), config);
        if (!scene.ok() || scene.status() != VX_OK) {
            std::fprintf(stderr, "scene creation failed: %s\n", vx_last_error());
            vx_ctx_destroy(ctx);
            return 1;
        }
        const size_t n = scene.size();
        size_t active = 0;
        for (uint8_t k : scene.kinematic) active += k ? 0 : 1;
        const size_t surface_count = NX * NY * NZ - (NX - 2) * (NY - 2) * (NZ - 2);
        struct Sample {
            size_t id, index, x, y, z;
        };
        std::vector<Sample> surface;
        surface.reserve(surface_count * 2 / 3 + 1);
        for (size_t z = 0; z < NZ; ++z)
            for (size_t y = 0; y < NY; ++y)
                for (size_t x = 0; x < NX; ++x) {
                    const size_t index = (z * NY + y) * NX + x;
                    const bool boundary = x == 0 || x + 1 == NX || y == 0 || y + 1 == NY || z == 0 || z + 1 == NZ;
                    if (boundary && index % 3 != 0) surface.push_back({surface.size(), index, x, y, z});
                }
        std::fprintf(stderr,
                     "solver scale capture: %zu REV, %zu active, %zu surface REV (%zu sampled), dt=%s s, substeps=%u, "
                     "steps=%zu, states=%zu, precision=%d\n",
                     n, active, surface_count, surface.size(), f32_display(config.fixed_dt).c_str(), config.substeps,
                     steps, saved_frames, config.precision);

        FILE* out = std::fopen(path.c_str(), "w");
        if (!out) {
            std::fprintf(stderr, "%s: cannot create\n", path.c_str());
            vx_ctx_destroy(ctx);
            return 1;
        }
        static char buffer[1 << 20];
        std::setvbuf(out, buffer, _IOFBF, sizeof buffer);
        std::fprintf(out, "H,%s,%zu,%zu\n", f32_display(config.fixed_dt).c_str(), steps, saved_frames);
        const auto clock = std::chrono::steady_clock::now();
        auto wall = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - clock).count(); };
        const unsigned __int128 intervals = saved_frames - 1;
        for (size_t frame = 0; frame <= steps; ++frame) {
            if (frame > 0) {
                const int32_t r = solver::step(scene);  // Scene::tick
                if (r != VX_OK && r != VX_NOT_CONVERGED) {
                    std::fprintf(stderr, "step %zu failed (%d): %s\n", frame, r, vx_last_error());
                    rc = 1;
                    break;
                }
            }
            if (frame % 10 == 0 || frame == steps)
                std::fprintf(stderr, "frame=%zu/%zu wall=%.2fs broken=%llu clusters=%zu residual=%.3e\n", frame, steps,
                             wall(), (unsigned long long)scene.broken, scene.cluster_count, scene.solver_residual);
            const bool save = frame == 0 || frame == steps ||
                              (frame * intervals / steps) > ((frame - 1) * intervals / steps);
            if (!save) continue;
            std::fprintf(out, "F,%zu,0,0,0,0,0,0,1,0,0,%llu,%zu,0\n", frame, (unsigned long long)scene.broken,
                         scene.cluster_count);
            const std::vector<std::array<double, 3>> pos = scene.positions();
            const std::vector<uint32_t> nbr = scene.neighbors();
            const std::vector<float> damage = scene.bond_damage();
            for (const Sample& s : surface) {
                float d;
                unsigned lost;
                surface_state(nbr, damage, n, s.x, s.y, s.z, d, lost);
                const std::array<double, 3>& p = pos[s.index];
                std::fprintf(out, "V,%zu,%zu,%s,%s,%s,%s,%u,%zu\n", frame, s.id, f32_display((float)p[0]).c_str(),
                             f32_display((float)p[1]).c_str(), f32_display((float)p[2]).c_str(),
                             f32_display(d).c_str(), lost, s.index);
            }
            std::fflush(out);
        }
        std::fclose(out);
        std::fprintf(stderr, "complete wall=%.2fs\n", wall());
    }
    vx_ctx_destroy(ctx);
    return rc;
}
