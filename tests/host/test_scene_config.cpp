// Scene configuration files: the RON loader of SceneConfig (src/scene.rs:215-307)
// and FractureConfig (src/fracture.rs:10-60) against the serde rules the
// reference derives (deny_unknown_fields, required fields, the two defaults)
// and its validation. Needs no GPU. Prints PASS/FAIL per test; exits non-zero
// on any failure. argv[1] (optional): a directory of RON scene files that
// must all load.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dirent.h>
#include <string>
#include <vector>

#include "vxsim_config.hpp"
#include "vxsim_materials.hpp"

using namespace vxsim;

static int g_failures = 0;
static bool g_ok = true;

#define CHECK(cond)                                                          \
    do {                                                                     \
        if (!(cond)) {                                                       \
            std::printf("  check failed at line %d: %s\n", __LINE__, #cond); \
            g_ok = false;                                                    \
        }                                                                    \
    } while (0)

static void run(const char* name, void (*fn)()) {
    g_ok = true;
    fn();
    std::printf("%s %s\n", g_ok ? "PASS" : "FAIL", name);
    std::fflush(stdout);
    if (!g_ok) ++g_failures;
}

// A complete file in the layout of the shipped scene files, with comments.
static const char* kFull = R"(// trunk chopping scene, Z up
(
    dimensions: (24, 20, 200), /* block comment /* nested */ still comment */
    branch_dimensions: (0, 0, 0),
    ground_dimensions: (64, 64, 1),
    tool_dimensions: (30, 4, 12),
    fibers: (0.0, 0.0, 1.0),
    anisotropy: 1.0,
    gravity: (0.0, 0.0, -9.81),
    fixed_dt: 0.016666668,
    substeps: 4,
    iterations: 60,
    solver_relative_tolerance: 0.00001,
    corotation_tolerance: 1e-5,
    corotation_iterations: 3,
    fracture: (
        damage_rate: 30.0,
        energy_release: 0.01,
        propagation_delay: 2,
        fatigue_cycles: 500.0,
        fatigue_exponent: 2.5,
        fatigue_threshold: 0.4,
        plastic_heat_fraction: 0.85,
        fragment_min_size: 8,
        cluster_interval: 5,
        friction: 0.3,
        restitution: 0.2,
    ),
    initial_speed: 6.5,
    tool_start: (-0.5, 0.0, 0.9),
)
)";

static std::string with(const std::string& base, const std::string& from, const std::string& to) {
    std::string s = base;
    const size_t at = s.find(from);
    if (at == std::string::npos) return "<pattern missing: " + from + ">";
    return s.replace(at, from.size(), to);
}

static bool parses(const std::string& text, SceneFileConfig& c, std::string& err) {
    return parse_scene_config(text, c, err);
}

static bool fails_with(const std::string& text, const char* fragment) {
    SceneFileConfig c;
    std::string err;
    if (parse_scene_config(text, c, err)) {
        std::printf("  parsed, expected an error containing `%s`\n", fragment);
        return false;
    }
    if (err.find(fragment) == std::string::npos) {
        std::printf("  error `%s` lacks `%s`\n", err.c_str(), fragment);
        return false;
    }
    return true;
}

static bool invalid(const std::string& text) {
    SceneFileConfig c;
    std::string err;
    if (!parse_scene_config(text, c, err)) {
        std::printf("  parse error %s\n", err.c_str());
        return false;
    }
    const char* why = c.validate();
    return why != nullptr && std::strcmp(why, "Invalid scene parameters") == 0;
}

static void full_file_reads_every_field() {
    SceneFileConfig c;
    std::string err;
    CHECK(parses(kFull, c, err));
    CHECK(err.empty());
    CHECK(c.dimensions[0] == 24 && c.dimensions[1] == 20 && c.dimensions[2] == 200);
    CHECK(c.branch_dimensions[0] == 0 && c.branch_dimensions[2] == 0);
    CHECK(c.ground_dimensions[0] == 64 && c.ground_dimensions[2] == 1);
    CHECK(c.tool_dimensions[0] == 30 && c.tool_dimensions[1] == 4 && c.tool_dimensions[2] == 12);
    CHECK(c.fibers[2] == 1.0f && c.anisotropy == 1.0f);
    CHECK(c.gravity[2] == -9.81f);
    CHECK(c.fixed_dt == 0.016666668f);  // the same f32 as Rust's parse
    CHECK(c.substeps == 4 && c.iterations == 60 && c.corotation_iterations == 3);
    CHECK(c.solver_relative_tolerance == 0.00001f && c.corotation_tolerance == 1e-5f);
    CHECK(c.fracture.damage_rate == 30.0f && c.fracture.energy_release == 0.01f);
    CHECK(c.fracture.propagation_delay == 2 && c.fracture.fragment_min_size == 8 && c.fracture.cluster_interval == 5);
    CHECK(c.fracture.fatigue_cycles == 500.0f && c.fracture.fatigue_exponent == 2.5f);
    CHECK(c.fracture.fatigue_threshold == 0.4f && c.fracture.plastic_heat_fraction == 0.85f);
    CHECK(c.fracture.friction == 0.3f && c.fracture.restitution == 0.2f);
    CHECK(c.initial_speed == 6.5f);
    CHECK(c.tool_start[0] == -0.5f && c.tool_start[2] == 0.9f);
    CHECK(c.validate() == nullptr);
}

// #[serde(default = "default_cuda_iterations")] and #[serde(default)]
static void omitted_fields_with_serde_defaults() {
    SceneFileConfig c;
    std::string err;
    CHECK(parses(kFull, c, err));
    CHECK(c.cuda_iterations == 160);
    CHECK(c.cpu_preconditioner == "incomplete_cholesky0");
    CHECK(parses(with(kFull, "    iterations: 60,", "    iterations: 60,\n    cuda_iterations: 320,\n"
                                                     "    cpu_preconditioner: block_jacobi,"),
                 c, err));
    CHECK(c.cuda_iterations == 320);
    CHECK(c.cpu_preconditioner == "block_jacobi");
    CHECK(fails_with(with(kFull, "    iterations: 60,", "    iterations: 60, cpu_preconditioner: jacobi,"),
                     "unknown variant `jacobi`"));
}

static void unknown_missing_and_duplicate_fields() {
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: 4,\n    sub_steps: 4,"), "unknown field `sub_steps`"));
    CHECK(fails_with(with(kFull, "    substeps: 4,\n", ""), "missing field `substeps`"));
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: 4, substeps: 5,"), "duplicate field `substeps`"));
    // FractureConfig has no defaults at all and denies unknown fields too
    CHECK(fails_with(with(kFull, "        friction: 0.3,\n", ""), "missing field `friction` in FractureConfig"));
    CHECK(fails_with(with(kFull, "        friction: 0.3,", "        friction: 0.3, drag: 1.0,"), "unknown field `drag`"));
    CHECK(fails_with(with(kFull, "    fracture: (", "    fracture: FractureSettings("), "expected struct FractureConfig"));
    CHECK(fails_with("()", "missing field `dimensions`"));
}

static void ron_syntax() {
    SceneFileConfig c;
    std::string err;
    // an explicit struct name, no trailing commas, integers for floats
    std::string named = with(kFull, "(\n    dimensions", "SceneConfig(\n    dimensions");
    named = with(named, "    tool_start: (-0.5, 0.0, 0.9),\n)", "    tool_start: (-1, 0, 1)\n)");
    CHECK(parses(named, c, err));
    CHECK(c.tool_start[0] == -1.0f && c.tool_start[2] == 1.0f);
    CHECK(fails_with(with(kFull, "(\n    dimensions", "Scene(\n    dimensions"), "expected struct SceneConfig"));
    // digit separators, hex integers, exponents
    CHECK(parses(with(kFull, "    iterations: 60,", "    iterations: 1_000,\n    cuda_iterations: 0x40,"), c, err));
    CHECK(c.iterations == 1000 && c.cuda_iterations == 64);
    CHECK(parses(with(kFull, "    fixed_dt: 0.016666668,", "    fixed_dt: 2.5E-3,"), c, err));
    CHECK(c.fixed_dt == 2.5e-3f);
    // integer fields reject floats and negatives; arrays need exactly 3 entries
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: 4.0,"), "expected usize"));
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: -4,"), "expected usize"));
    CHECK(fails_with(with(kFull, "    fibers: (0.0, 0.0, 1.0),", "    fibers: (0.0, 1.0),"), "invalid length 2"));
    CHECK(fails_with(with(kFull, "    anisotropy: 1.0,", "    anisotropy: one,"), "expected f32"));
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: 99999999999999999999999,"), "out of range"));
    // syntax errors carry line:column
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps 4,"), "expected ':' after field `substeps`"));
    CHECK(fails_with(std::string(kFull) + " )", "trailing characters"));
    CHECK(fails_with("( dimensions: (1, 2, 3) /* open", "unterminated block comment"));
    CHECK(fails_with(with(kFull, "    substeps: 4,", "    substeps: 4 iterations: 3,"), "expected ',' or ')'"));
    std::string e;
    CHECK(!parse_scene_config(with(kFull, "    substeps: 4,", "    substeps 4,"), c, e));
    CHECK(e.rfind("11:", 0) == 0);  // line 11 of the file
}

// SceneConfig::validate (src/scene.rs:275-297) and FractureConfig::validate
// (src/fracture.rs:45-60): each rule on its own.
static void validation_rules() {
    const std::string f = kFull;
    CHECK(invalid(with(f, "dimensions: (24, 20, 200)", "dimensions: (24, 0, 200)")));
    CHECK(invalid(with(f, "ground_dimensions: (64, 64, 1)", "ground_dimensions: (64, 64, 0)")));
    CHECK(invalid(with(f, "tool_dimensions: (30, 4, 12)", "tool_dimensions: (30, 1, 12)")));
    CHECK(invalid(with(f, "anisotropy: 1.0", "anisotropy: 1.5")));
    CHECK(invalid(with(f, "anisotropy: 1.0", "anisotropy: -0.1")));
    CHECK(invalid(with(f, "gravity: (0.0, 0.0, -9.81)", "gravity: (0.0, inf, -9.81)")));
    CHECK(invalid(with(f, "tool_start: (-0.5, 0.0, 0.9)", "tool_start: (NaN, 0.0, 0.9)")));
    CHECK(invalid(with(f, "initial_speed: 6.5", "initial_speed: -1.0")));
    CHECK(invalid(with(f, "fibers: (0.0, 0.0, 1.0)", "fibers: (0.0, 0.0, 0.00001)")));  // |f|^2 < 1e-8
    CHECK(invalid(with(f, "fixed_dt: 0.016666668", "fixed_dt: 0.0")));
    CHECK(invalid(with(f, "substeps: 4", "substeps: 0")));
    CHECK(invalid(with(f, "iterations: 60", "iterations: 0")));
    CHECK(invalid(with(f, "iterations: 60,", "iterations: 60, cuda_iterations: 0,")));
    CHECK(invalid(with(f, "corotation_iterations: 3", "corotation_iterations: 0")));
    CHECK(invalid(with(f, "solver_relative_tolerance: 0.00001", "solver_relative_tolerance: 0.0")));
    CHECK(invalid(with(f, "corotation_tolerance: 1e-5", "corotation_tolerance: -1e-5")));
    CHECK(invalid(with(f, "damage_rate: 30.0", "damage_rate: 0.0")));
    CHECK(invalid(with(f, "energy_release: 0.01", "energy_release: 1.01")));
    CHECK(invalid(with(f, "fatigue_cycles: 500.0", "fatigue_cycles: 0.0")));
    CHECK(invalid(with(f, "fatigue_exponent: 2.5", "fatigue_exponent: 0.5")));
    CHECK(invalid(with(f, "fatigue_threshold: 0.4", "fatigue_threshold: 1.0")));  // [0, 1)
    CHECK(invalid(with(f, "plastic_heat_fraction: 0.85", "plastic_heat_fraction: 1.1")));
    CHECK(invalid(with(f, "fragment_min_size: 8", "fragment_min_size: 0")));
    CHECK(invalid(with(f, "cluster_interval: 5", "cluster_interval: 0")));
    CHECK(invalid(with(f, "friction: 0.3", "friction: -0.1")));
    CHECK(invalid(with(f, "restitution: 0.2", "restitution: 2.0")));
    // the boundaries that stay valid
    SceneFileConfig c;
    std::string err;
    CHECK(parses(with(with(with(f, "anisotropy: 1.0", "anisotropy: 0.0"), "energy_release: 0.01", "energy_release: 1.0"),
                      "fatigue_threshold: 0.4", "fatigue_threshold: 0.0"),
                 c, err));
    CHECK(c.validate() == nullptr);
    CHECK(parses(with(f, "fibers: (0.0, 0.0, 1.0)", "fibers: (0.0, 0.0, 0.0002)"), c, err));
    CHECK(c.validate() == nullptr);  // 4e-8 >= 1e-8
}

static void defaults_match_the_reference() {
    const SceneFileConfig d;  // SceneConfig::default, src/scene.rs:238-262
    CHECK(d.validate() == nullptr);
    CHECK(d.fixed_dt == 0.001f && d.substeps == 4 && d.iterations == 80 && d.cuda_iterations == 160);
    CHECK(d.corotation_iterations == 2 && d.solver_relative_tolerance == 1e-5f);
    const FractureSettings f;  // FractureConfig::default, src/fracture.rs:27-42
    CHECK(f.validate());
    CHECK(f.damage_rate == 35.0f && f.energy_release == 0.005f && f.propagation_delay == 1);
    CHECK(f.fatigue_cycles == 1000.0f && f.fatigue_exponent == 3.0f && f.fatigue_threshold == 0.5f);
    CHECK(f.plastic_heat_fraction == 0.9f && f.fragment_min_size == 10 && f.cluster_interval == 10);
}

static void solver_settings_follow_the_file() {
    SceneFileConfig c;
    std::string err;
    CHECK(parses(kFull, c, err));
    const SceneConfig s = c.solver_config();
    CHECK(s.fixed_dt == 0.016666668f && s.substeps == 4);
    CHECK(s.iterations == 160);  // the device path's cap is cuda_iterations
    CHECK(s.corotation_iterations == 3 && s.corotation_tolerance == 1e-5f);
    CHECK(s.gravity[2] == -9.81f);
    CHECK(s.fracture);
    CHECK(s.fracture_config.damage_rate == 30.0 && s.fracture_config.energy_release == (double)0.01f);
    CHECK(s.fracture_config.plastic_heat_fraction == (double)0.85f);
    CHECK(s.contact && s.restitution == 0.2f && s.friction == 0.3f);
    // the mirror's defaults equal FractureConfig::default's f32 values
    const SceneConfig d;
    const SceneConfig from_default = SceneFileConfig{}.solver_config();
    CHECK(std::memcmp(&d.fracture_config, &from_default.fracture_config, sizeof(vx_fracture_config)) == 0);
}

static void material_table_lookup() {
    const std::vector<vx_material> t = builtin_materials();
    CHECK(t.size() == 10);
    CHECK(material_component_id("iron") == 2 && material_component_id("Wood") == 1);
    CHECK(material_component_id("unobtainium") == -1);
    CHECK(t[2].density == 7870.f && t[2].young == 200e9f && t[2].fracture_mode == VX_DUCTILE);
    CHECK(t[1].compressive_strength_perp == 2e6f && t[1].fracture_mode == VX_MIXED);
}

static void load_directory(const char* dir) {
    DIR* d = opendir(dir);
    if (!d) {
        std::printf("FAIL cannot open %s\n", dir);
        ++g_failures;
        return;
    }
    std::vector<std::string> files;
    while (dirent* e = readdir(d)) {
        const std::string name = e->d_name;
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".ron") == 0) files.push_back(name);
    }
    closedir(d);
    for (const std::string& name : files) {
        SceneFileConfig c;
        std::string err;
        const bool ok = load_scene_config(std::string(dir) + "/" + name, c, err);
        std::printf("%s load %s%s%s\n", ok ? "PASS" : "FAIL", name.c_str(), ok ? "" : ": ", err.c_str());
        if (!ok) ++g_failures;
    }
}

int main(int argc, char** argv) {
    run("full_file_reads_every_field", full_file_reads_every_field);
    run("omitted_fields_with_serde_defaults", omitted_fields_with_serde_defaults);
    run("unknown_missing_and_duplicate_fields", unknown_missing_and_duplicate_fields);
    run("ron_syntax", ron_syntax);
    run("validation_rules", validation_rules);
    run("defaults_match_the_reference", defaults_match_the_reference);
    run("solver_settings_follow_the_file", solver_settings_follow_the_file);
    run("material_table_lookup", material_table_lookup);
    if (argc > 1) load_directory(argv[1]);
    std::printf("%d failures\n", g_failures);
    return g_failures ? 1 : 0;
}
