"""Built-in material table of the elastic solve.

The values are those of ``Material::table`` in the reference
(src/material.rs:73-342, including the per-row overrides at :274-320); only
the fields that the stiffness law (tensor_compliance, src/solver.rs:37-63),
the thermal rest length (:78-95) and the limit law (pair_limits,
src/fracture.rs:76-133) read are kept, plus what ``thermal_strength_scale``
and ``phase_state`` need at a given temperature (src/material.rs:485-565).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

BRITTLE, DUCTILE, MIXED = 0, 1, 2
INF = math.inf

# numpy layout of ``vx_material`` in include/vxcorot.h (17 f32 + one i32).
MATERIAL_DTYPE = np.dtype(
    [
        ("density", "<f4"),
        ("young", "<f4"),
        ("young_perp", "<f4"),
        ("shear", "<f4"),
        ("tensile_strength", "<f4"),
        ("tensile_strength_perp", "<f4"),
        ("compressive_strength", "<f4"),
        ("compressive_strength_perp", "<f4"),
        ("shear_strength", "<f4"),
        ("shear_strength_perp", "<f4"),
        ("yield_strength", "<f4"),
        ("hardening_modulus", "<f4"),
        ("failure_plastic_strain", "<f4"),
        ("fracture_energy", "<f4"),
        ("fracture_energy_perp", "<f4"),
        ("thermal_expansion_parallel", "<f4"),
        ("thermal_expansion_perpendicular", "<f4"),
        ("fracture_mode", "<i4"),
    ]
)


@dataclass(frozen=True)
class Material:
    name: str
    density: float
    young: float
    young_perp: float
    shear: float
    tensile_strength: float
    tensile_strength_perp: float
    compressive_strength: float
    compressive_strength_perp: float
    shear_strength: float
    shear_strength_perp: float
    yield_strength: float
    hardening_modulus: float = 0.0
    failure_plastic_strain: float = 0.0
    fracture_energy: float = 0.0
    fracture_energy_perp: float = 0.0
    thermal_expansion_parallel: float = 0.0
    thermal_expansion_perpendicular: float = 0.0
    fracture_mode: int = BRITTLE
    heat_capacity: float = 1.0
    melt_temp: float = INF
    strength_softening_start_ratio: float = 1.0
    boil_temp: float = INF
    latent_fusion: float = 0.0
    latent_vaporization: float = 0.0

    def record(self) -> np.void:
        rec = np.zeros((), dtype=MATERIAL_DTYPE)
        for field in MATERIAL_DTYPE.names:
            rec[field] = getattr(self, field)
        return rec

    def thermal_strength_scale(self, temperature: float) -> float:
        """Pre-melt strength factor (src/material.rs:485-501)."""
        r = self.strength_softening_start_ratio
        if (
            not math.isfinite(temperature)
            or not math.isfinite(self.melt_temp)
            or self.melt_temp <= 0.0
            or not math.isfinite(r)
            or not (0.0 <= r < 1.0)
        ):
            return 1.0
        onset = self.melt_temp * r
        if temperature <= onset:
            return 1.0
        return min(max((self.melt_temp - temperature) / (self.melt_temp - onset), 0.0), 1.0)

    def solid_fraction(self, temperature: float) -> float:
        """Solid fraction at a temperature below boiling (src/material.rs:518-565).

        Only the solid/melting branch matters for the elastic solve: a REV at
        or above its melting point carries no solid fraction.
        """
        if math.isfinite(self.melt_temp) and temperature >= self.melt_temp:
            return 0.0
        return 1.0


def _new(name, density, young, young_perp, shear, tensile, tensile_perp, compressive,
         shear_strength, yield_strength, heat_capacity, melt, gc, gc_perp, boil, lf, lv):
    # Material::new (src/material.rs:344-396): perpendicular compression and
    # shear default to their parallel values; brittle; no hardening.
    return Material(
        name=name, density=density, young=young, young_perp=young_perp, shear=shear,
        tensile_strength=tensile, tensile_strength_perp=tensile_perp,
        compressive_strength=compressive, compressive_strength_perp=compressive,
        shear_strength=shear_strength, shear_strength_perp=shear_strength,
        yield_strength=yield_strength, fracture_energy=gc, fracture_energy_perp=gc_perp,
        heat_capacity=heat_capacity, melt_temp=melt, boil_temp=boil,
        latent_fusion=lf, latent_vaporization=lv,
    )


def table() -> list[Material]:
    """The reference's ten built-in components in table order."""
    t = [
        _new("air", 1.225, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1005.0, INF, 0.0, 0.0, INF, 0.0, 0.0),
        _new("wood", 650.0, 10e9, 0.6e9, 0.65e9, 100e6, 2.5e6, 50e6, 12e6, 25e6, 1700.0, INF, 350.0, 80.0, INF, 0.0, 0.0),
        _new("iron", 7870.0, 200e9, 200e9, 77e9, 350e6, 350e6, 350e6, 200e6, 200e6, 450.0, 1811.0, 30000.0, 30000.0, 3134.0, 247_000.0, 6_300_000.0),
        _new("stone", 2700.0, 50e9, 50e9, 20e9, 7e6, 7e6, 120e6, 12e6, 100e6, 790.0, 1500.0, 80.0, 80.0, INF, 300_000.0, 0.0),
        _new("water", 1000.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 4184.0, 273.15, 0.0, 0.0, 373.15, 333_500.0, 2_256_000.0),
        _new("aluminum", 2700.0, 69e9, 69e9, 26e9, 310e6, 310e6, 310e6, 180e6, 276e6, 897.0, 933.15, 15_000.0, 15_000.0, 2743.0, 397_000.0, 10_500_000.0),
        _new("copper", 8960.0, 117e9, 117e9, 44e9, 220e6, 220e6, 210e6, 120e6, 70e6, 385.0, 1357.77, 30_000.0, 30_000.0, 2835.0, 205_000.0, 4_730_000.0),
        _new("glass", 2500.0, 70e9, 70e9, 29e9, 45e6, 45e6, 1000e6, 35e6, 45e6, 840.0, 1700.0, 10.0, 10.0, INF, 0.0, 0.0),
        _new("concrete", 2400.0, 30e9, 30e9, 12.5e9, 3.5e6, 3.5e6, 40e6, 5e6, 3.5e6, 880.0, 1773.0, 100.0, 100.0, INF, 0.0, 0.0),
        _new("rubber", 1100.0, 10e6, 10e6, 3.3e6, 20e6, 20e6, 20e6, 10e6, 5e6, 1900.0, INF, 5_000.0, 5_000.0, INF, 0.0, 0.0),
    ]
    # Row overrides, src/material.rs:274-320.
    t[1] = replace(t[1], fracture_mode=MIXED, thermal_expansion_parallel=3.0e-6,
                   thermal_expansion_perpendicular=30.0e-6, compressive_strength_perp=2e6,
                   shear_strength_perp=3e6, hardening_modulus=2e9, failure_plastic_strain=0.04)
    t[2] = replace(t[2], fracture_mode=DUCTILE, thermal_expansion_parallel=12.0e-6,
                   thermal_expansion_perpendicular=12.0e-6, strength_softening_start_ratio=0.7,
                   hardening_modulus=1e9, failure_plastic_strain=0.15)
    t[5] = replace(t[5], fracture_mode=DUCTILE, thermal_expansion_parallel=23.0e-6,
                   thermal_expansion_perpendicular=23.0e-6, strength_softening_start_ratio=0.7,
                   hardening_modulus=0.7e9, failure_plastic_strain=0.18)
    t[6] = replace(t[6], fracture_mode=DUCTILE, thermal_expansion_parallel=16.5e-6,
                   thermal_expansion_perpendicular=16.5e-6, strength_softening_start_ratio=0.7,
                   hardening_modulus=0.45e9, failure_plastic_strain=0.30)
    t[7] = replace(t[7], strength_softening_start_ratio=0.7, thermal_expansion_parallel=9.0e-6,
                   thermal_expansion_perpendicular=9.0e-6)
    t[8] = replace(t[8], strength_softening_start_ratio=0.7, thermal_expansion_parallel=10.0e-6,
                   thermal_expansion_perpendicular=10.0e-6)
    t[3] = replace(t[3], thermal_expansion_parallel=8.0e-6, thermal_expansion_perpendicular=8.0e-6)
    t[4] = replace(t[4], thermal_expansion_parallel=69.0e-6, thermal_expansion_perpendicular=69.0e-6)
    t[9] = replace(t[9], fracture_mode=DUCTILE, thermal_expansion_parallel=100.0e-6,
                   thermal_expansion_perpendicular=100.0e-6, hardening_modulus=20e6,
                   failure_plastic_strain=1.0)
    return t


def component_id(name: str) -> int:
    for i, m in enumerate(table()):
        if m.name.lower() == name.lower():
            return i
    raise KeyError(name)


def records(materials: list[Material]) -> np.ndarray:
    out = np.zeros(len(materials), dtype=MATERIAL_DTYPE)
    for i, m in enumerate(materials):
        out[i] = m.record()
    return out
