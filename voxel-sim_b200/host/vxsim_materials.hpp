// vxsim_materials.hpp — the built-in material table (Material::table,
// src/material.rs:73-342, with the per-row overrides of :274-320), reduced to
// the vx_material fields the elastic solve and the fracture law read, and
// Material::component_id (lookup by name, case-insensitive).
#pragma once

#include <cstring>
#include <string>
#include <strings.h>
#include <vector>

#include "../../include/vxcorot.h"

namespace vxsim {

inline const char* const kMaterialNames[10] = {"air",      "wood",   "iron",  "stone",    "water",
                                               "aluminum", "copper", "glass", "concrete", "rubber"};

inline std::vector<vx_material> builtin_materials() {
    // Material::new (src/material.rs:344-396): perpendicular compression and
    // shear equal their parallel values; brittle; no hardening.
    auto row = [](float density, float young, float young_perp, float shear, float tensile, float tensile_perp,
                  float compressive, float shear_strength, float yield, float gc, float gc_perp) {
        vx_material m{};
        m.density = density;
        m.young = young;
        m.young_perp = young_perp;
        m.shear = shear;
        m.tensile_strength = tensile;
        m.tensile_strength_perp = tensile_perp;
        m.compressive_strength = compressive;
        m.compressive_strength_perp = compressive;
        m.shear_strength = shear_strength;
        m.shear_strength_perp = shear_strength;
        m.yield_strength = yield;
        m.fracture_energy = gc;
        m.fracture_energy_perp = gc_perp;
        m.fracture_mode = VX_BRITTLE;
        return m;
    };
    std::vector<vx_material> t = {
        row(1.225f, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
        row(650.f, 10e9f, 0.6e9f, 0.65e9f, 100e6f, 2.5e6f, 50e6f, 12e6f, 25e6f, 350.f, 80.f),
        row(7870.f, 200e9f, 200e9f, 77e9f, 350e6f, 350e6f, 350e6f, 200e6f, 200e6f, 30000.f, 30000.f),
        row(2700.f, 50e9f, 50e9f, 20e9f, 7e6f, 7e6f, 120e6f, 12e6f, 100e6f, 80.f, 80.f),
        row(1000.f, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
        row(2700.f, 69e9f, 69e9f, 26e9f, 310e6f, 310e6f, 310e6f, 180e6f, 276e6f, 15000.f, 15000.f),
        row(8960.f, 117e9f, 117e9f, 44e9f, 220e6f, 220e6f, 210e6f, 120e6f, 70e6f, 30000.f, 30000.f),
        row(2500.f, 70e9f, 70e9f, 29e9f, 45e6f, 45e6f, 1000e6f, 35e6f, 45e6f, 10.f, 10.f),
        row(2400.f, 30e9f, 30e9f, 12.5e9f, 3.5e6f, 3.5e6f, 40e6f, 5e6f, 3.5e6f, 100.f, 100.f),
        row(1100.f, 10e6f, 10e6f, 3.3e6f, 20e6f, 20e6f, 20e6f, 10e6f, 5e6f, 5000.f, 5000.f),
    };
    auto expansion = [&t](int k, float a) {
        t[k].thermal_expansion_parallel = a;
        t[k].thermal_expansion_perpendicular = a;
    };
    // wood
    t[1].fracture_mode = VX_MIXED;
    t[1].thermal_expansion_parallel = 3.0e-6f;
    t[1].thermal_expansion_perpendicular = 30.0e-6f;
    t[1].compressive_strength_perp = 2e6f;
    t[1].shear_strength_perp = 3e6f;
    t[1].hardening_modulus = 2e9f;
    t[1].failure_plastic_strain = 0.04f;
    // metals
    t[2].fracture_mode = VX_DUCTILE;
    expansion(2, 12.0e-6f);
    t[2].hardening_modulus = 1e9f;
    t[2].failure_plastic_strain = 0.15f;
    t[5].fracture_mode = VX_DUCTILE;
    expansion(5, 23.0e-6f);
    t[5].hardening_modulus = 0.7e9f;
    t[5].failure_plastic_strain = 0.18f;
    t[6].fracture_mode = VX_DUCTILE;
    expansion(6, 16.5e-6f);
    t[6].hardening_modulus = 0.45e9f;
    t[6].failure_plastic_strain = 0.30f;
    expansion(7, 9.0e-6f);
    expansion(8, 10.0e-6f);
    expansion(3, 8.0e-6f);
    expansion(4, 69.0e-6f);
    t[9].fracture_mode = VX_DUCTILE;
    expansion(9, 100.0e-6f);
    t[9].hardening_modulus = 20e6f;
    t[9].failure_plastic_strain = 1.0f;
    return t;
}

// Material::component_id: the table index of a name, or -1.
inline int material_component_id(const std::string& name) {
    for (int k = 0; k < 10; ++k)
        if (strcasecmp(name.c_str(), kMaterialNames[k]) == 0) return k;
    return -1;
}

}  // namespace vxsim
