"""ctypes binding of the CPU oracle (oracle/vx_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the package smoke check and the
bench's CPU-baseline arm, as the checker. Never imported by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
VXO_CELL = float(np.float32(0.01))
VXO_AREA = float(np.float32(np.float32(0.01) * np.float32(0.01)))
LIB_PATH = HERE / "build" / "liboracle.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)


class VxMaterial(C.Structure):
    _fields_ = [(name, C.c_float) for name in (
        "density", "young", "young_perp", "shear", "tensile_strength", "tensile_strength_perp",
        "compressive_strength", "compressive_strength_perp", "shear_strength", "shear_strength_perp",
        "yield_strength", "hardening_modulus", "failure_plastic_strain", "fracture_energy",
        "fracture_energy_perp", "thermal_expansion_parallel", "thermal_expansion_perpendicular")] + [
        ("fracture_mode", C.c_int32)]


class VxoScene(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("pos", f64p), ("rot", f64p), ("kinematic", u8p), ("mass", f64p),
        ("material", u32p), ("materials", C.POINTER(VxMaterial)), ("fiber", f64p),
        ("anisotropy", f64p), ("solid", f64p), ("thermal_scale", f64p), ("thermal_delta", f64p),
        ("nbr", u32p), ("formation", f64p), ("plastic", f64p), ("damage", f64p),
        ("eq_plastic", f64p),
    ]


class VxoSystem(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("free", f64p), ("diag", f64p), ("rhs", f64p), ("k", f64p),
        ("material_k", f64p), ("frame", f64p), ("rest", f64p), ("state", u8p), ("c_i", u32p),
        ("c_j", u32p), ("c_axis", u32p), ("c_count", C.c_uint32), ("incidence", u32p),
        ("incidence_len", u8p), ("partner", u32p),
    ]


class VxoLimits(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "tension", "compression", "shear", "yield_stress", "hardening", "plastic_failure",
        "ductility", "fracture_energy")]


class VxoFractureConfig(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "damage_rate", "energy_release", "fatigue_cycles", "fatigue_exponent",
        "fatigue_threshold", "plastic_heat_fraction")]


class VxoBond(C.Structure):
    _fields_ = [("neighbor", C.c_uint32), ("formation", C.c_double * 3), ("plastic", C.c_double * 3)] + [
        (k, C.c_double) for k in ("damage", "equivalent_plastic_strain", "plastic_work", "fatigue_damage",
                                  "previous_stress_ratio", "reversal_stress_ratio", "loading_increment")]


class VxoDissipation(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("plastic_heat", "stored_plastic", "surface_work", "damage_heat", "released")]

    def total(self):
        return self.plastic_heat + self.stored_plastic + self.surface_work + self.damage_heat + self.released


class VxoStepConfig(C.Structure):
    _fields_ = [
        ("fixed_dt", C.c_double), ("substeps", C.c_uint32), ("iterations", C.c_uint32),
        ("solver_tolerance", C.c_double), ("corotation_tolerance", C.c_double),
        ("corotation_iterations", C.c_uint32), ("gravity", C.c_double * 3),
        ("fracture", VxoFractureConfig), ("fracture_enabled", C.c_int),
        ("contact_enabled", C.c_int), ("restitution", C.c_double), ("friction", C.c_double),
    ]


class VxoDynamics(C.Structure):
    _fields_ = [
        ("velocity", f64p), ("previous", f64p), ("target_mask", u8p), ("target", f64p),
        ("applied_loads", f64p), ("bonds", C.POINTER(VxoBond)), ("last_force", f64p),
        ("solver_residual", C.c_double), ("broken", C.c_uint64), ("pcg_iterations", C.c_uint64),
        ("external_work", C.c_double), ("plastic_heat", C.c_double), ("stored_plastic", C.c_double),
        ("surface_work", C.c_double), ("damage_heat", C.c_double), ("pending_release", C.c_double),
        ("rest", f64p), ("contacts", C.c_uint64), ("restitution_heat", C.c_double), ("friction_heat", C.c_double),
    ]


class VxoContact(C.Structure):
    _fields_ = [("i", C.c_uint32), ("j", C.c_uint32), ("normal", C.c_int32), ("new_impact", C.c_int32),
                ("order", C.c_uint32)]


class VxoContactStats(C.Structure):
    _fields_ = [("candidates", C.c_uint64), ("pairs", C.c_uint64), ("contacts", C.c_uint64), ("sweeps", C.c_uint32)]


def default_fracture_config() -> VxoFractureConfig:
    """FractureConfig::default / scenes/wood_chop.ron (src/fracture.rs:27-42)."""
    return VxoFractureConfig(35.0, 0.005, 1000.0, 3.0, 0.5, 0.9)


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.vxo_fit_rotations.restype = C.c_double
        L.vxo_fit_rotations.argtypes = [C.POINTER(VxoScene)]
        L.vxo_build_topology.restype = C.c_uint32
        L.vxo_build_topology.argtypes = [i32p, u8p, C.c_uint32, u32p]
        L.vxo_system_alloc.argtypes = [C.POINTER(VxoSystem), C.c_uint32]
        L.vxo_system_free.argtypes = [C.POINTER(VxoSystem)]
        L.vxo_assemble.argtypes = [C.POINTER(VxoScene), u8p, f64p, f64p, C.c_double, C.POINTER(VxoSystem)]
        L.vxo_matvec.argtypes = [C.POINTER(VxoSystem), f64p, f64p]
        L.vxo_factor_block_jacobi.argtypes = [C.POINTER(VxoSystem), f64p]
        L.vxo_pcg.argtypes = [C.POINTER(VxoSystem), f64p, C.c_uint32, C.c_double, C.c_int, f64p, u32p, f64p]
        L.vxo_true_residual.restype = C.c_double
        L.vxo_true_residual.argtypes = [C.POINTER(VxoSystem), f64p]
        L.vxo_solve_coupled.argtypes = [C.POINTER(VxoScene), u8p, f64p, f64p, C.c_double, C.c_uint32,
                                        C.c_double, C.c_int, f64p, C.POINTER(VxoSystem), u32p, f64p]
        L.vxo_bond_stress.argtypes = [C.POINTER(VxoScene), C.POINTER(VxoSystem), f64p, f64p]
        L.vxo_make_constraint.argtypes = [C.POINTER(VxoScene), C.c_uint32, C.c_int, C.c_uint32, f64p, f64p, f64p, f64p]
        L.vxo_stiffness_matrix.argtypes = [C.POINTER(VxoScene), C.c_uint32, C.c_uint32, f64p, f64p]
        L.vxo_bond_thermal_rest.argtypes = [C.POINTER(VxoScene), C.c_uint32, C.c_uint32, f64p, f64p]
        L.vxo_basis.argtypes = [C.c_int, f64p, f64p]
        L.vxo_slerp_half.argtypes = [f64p, f64p, f64p]
        L.vxo_quat_from_mat3.argtypes = [f64p, f64p]
        L.vxo_pair_limits.argtypes = [C.POINTER(VxMaterial), C.POINTER(VxMaterial), f64p, f64p, C.POINTER(VxoLimits)]
        L.vxo_bond_limits.argtypes = [C.POINTER(VxoScene), C.c_uint32, C.c_uint32, f64p, C.POINTER(VxoLimits)]
        L.vxo_fracture_update.argtypes = [C.POINTER(VxoBond), f64p, f64p, C.POINTER(VxoLimits), C.c_double,
                                          C.POINTER(VxoFractureConfig), C.POINTER(VxoDissipation)]
        L.vxo_fatigue.argtypes = [C.POINTER(VxoBond), C.c_double, C.POINTER(VxoFractureConfig)]
        L.vxo_stress_ratio.restype = C.c_double
        L.vxo_stress_ratio.argtypes = [f64p, f64p, f64p, C.POINTER(VxoLimits), C.c_double]
        L.vxo_pack_rows.restype = C.c_uint32
        L.vxo_pack_rows.argtypes = [C.POINTER(VxoSystem), u32p, f32p, u32p, f32p, f32p, f32p]
        L.vxo_pcg_rows_f32.argtypes = [C.c_uint32, f32p, u32p, f32p, f32p, C.c_uint32, C.c_float, C.c_int,
                                       f32p, u32p, f32p]
        L.vxo_cuda_pcg_emulate.argtypes = [C.c_uint32, f32p, u32p, f32p, f32p, f32p, C.c_uint32, C.c_float,
                                           f32p, u32p, f32p]
        L.vxo_step.argtypes = [C.POINTER(VxoScene), C.POINTER(VxoStepConfig), C.POINTER(VxoDynamics)]
        L.vxo_contact_project.restype = C.c_uint32
        L.vxo_contact_project.argtypes = [C.c_uint32, f64p, f64p, f64p, u8p, f64p, u8p, u32p,
                                          C.POINTER(C.POINTER(VxoContact)), C.POINTER(VxoContactStats)]
        L.vxo_resolve_velocities.argtypes = [C.c_uint32, f64p, f64p, u8p, f64p, u8p, C.POINTER(VxoContact),
                                             C.c_uint32, C.c_double, C.c_double, f64p, f64p]
        L.vxo_contact_box.argtypes = [f64p, f64p, C.c_uint32, i32p, i32p]
        L.vxo_local_continuum_pair.restype = C.c_int
        L.vxo_local_continuum_pair.argtypes = [f64p, u32p, C.c_uint32, C.c_uint32]
        L.free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def ptr(a: np.ndarray, ctype):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def material_struct(m) -> VxMaterial:
    out = VxMaterial()
    for name, _ in VxMaterial._fields_:
        setattr(out, name, getattr(m, name))
    return out


class OracleScene:
    """Double-precision copy of a vxsim Scene wired into a ``vxo_scene``."""

    def __init__(self, scene):
        n = scene.n
        self.scene = scene
        self.n = n
        self.pos = np.ascontiguousarray(scene.position, np.float64).reshape(-1).copy()
        self.rot = np.ascontiguousarray(scene.rotation, np.float64).reshape(-1).copy()
        self.kin = np.ascontiguousarray(scene.kinematic, np.uint8).copy()
        self.mass = scene.mass.astype(np.float64)
        self.material = np.ascontiguousarray(scene.material, np.uint32)
        self.mats = (VxMaterial * len(scene.materials))(*[material_struct(m) for m in scene.materials])
        self.fiber = scene.fiber.astype(np.float64).reshape(-1).copy()
        self.aniso = scene.anisotropy.astype(np.float64)
        self.solid = scene.solid_fraction.astype(np.float64)
        self.tscale = scene.thermal_strength.astype(np.float64)
        self.tdelta = scene.thermal_delta.astype(np.float64)
        self.nbr = np.ascontiguousarray(scene.neighbor, np.uint32).reshape(-1).copy()
        self.formation = scene.formation_offset.astype(np.float64).reshape(-1).copy()
        self.plastic = scene.plastic_strain.astype(np.float64).reshape(-1).copy()
        self.damage = scene.damage.astype(np.float64).reshape(-1).copy()
        self.eqp = scene.equivalent_plastic.astype(np.float64).reshape(-1).copy()
        self.s = VxoScene(
            n, ptr(self.pos, C.c_double), ptr(self.rot, C.c_double), ptr(self.kin, C.c_uint8),
            ptr(self.mass, C.c_double), ptr(self.material, C.c_uint32), self.mats,
            ptr(self.fiber, C.c_double), ptr(self.aniso, C.c_double), ptr(self.solid, C.c_double),
            ptr(self.tscale, C.c_double), ptr(self.tdelta, C.c_double), ptr(self.nbr, C.c_uint32),
            ptr(self.formation, C.c_double), ptr(self.plastic, C.c_double), ptr(self.damage, C.c_double),
            ptr(self.eqp, C.c_double))
        self.target_mask = np.ascontiguousarray(scene.target_mask, np.uint8).copy()
        self.loads = np.ascontiguousarray(scene.loads, np.float64).reshape(-1).copy()
        self.sys = VxoSystem()
        lib().vxo_system_alloc(C.byref(self.sys), n)
        self.factor = np.zeros(9 * max(n, 1), np.float64)

    def __del__(self):
        try:
            lib().vxo_system_free(C.byref(self.sys))
        except Exception:
            pass

    # -- views of the assembled system --------------------------------------
    def system_arrays(self):
        n = self.n
        s = self.sys
        as_np = lambda p, cnt, dt: np.ctypeslib.as_array(p, shape=(cnt,)).copy()
        return dict(
            free=as_np(s.free, 3 * n, np.float64).reshape(n, 3),
            diag=as_np(s.diag, 9 * n, np.float64).reshape(n, 3, 3),
            rhs=as_np(s.rhs, 3 * n, np.float64).reshape(n, 3),
            k=as_np(s.k, 27 * n, np.float64).reshape(3, n, 3, 3),
            material_k=as_np(s.material_k, 27 * n, np.float64).reshape(3, n, 3, 3),
            frame=as_np(s.frame, 27 * n, np.float64).reshape(3, n, 3, 3),
            rest=as_np(s.rest, 9 * n, np.float64).reshape(3, n, 3),
            state=as_np(s.state, 3 * n, np.uint8).reshape(3, n),
        )

    def positions(self):
        return self.pos.reshape(-1, 3).copy()

    def rotations(self):
        return self.rot.reshape(-1, 4).copy()

    def fit_rotations(self) -> float:
        return lib().vxo_fit_rotations(C.byref(self.s))

    def assemble(self, h, predicted=None):
        pred = None if predicted is None else np.ascontiguousarray(predicted, np.float64).reshape(-1)
        lib().vxo_assemble(C.byref(self.s), ptr(self.target_mask, C.c_uint8), ptr(self.loads, C.c_double),
                           None if pred is None else ptr(pred, C.c_double), h, C.byref(self.sys))

    def matvec(self, p):
        p = np.ascontiguousarray(p, np.float64).reshape(-1)
        out = np.zeros_like(p)
        lib().vxo_matvec(C.byref(self.sys), ptr(p, C.c_double), ptr(out, C.c_double))
        return out.reshape(-1, 3)

    def factor_block_jacobi(self):
        lib().vxo_factor_block_jacobi(C.byref(self.sys), ptr(self.factor, C.c_double))

    def pcg(self, max_iterations, tolerance, fixed_iterations=False):
        dx = np.zeros(3 * self.n, np.float64)
        it = C.c_uint32()
        res = C.c_double()
        lib().vxo_pcg(C.byref(self.sys), ptr(self.factor, C.c_double), max_iterations, tolerance,
                      int(fixed_iterations), ptr(dx, C.c_double), C.byref(it), C.byref(res))
        return dx.reshape(-1, 3), it.value, res.value

    def true_residual(self, dx):
        dx = np.ascontiguousarray(dx, np.float64).reshape(-1)
        return lib().vxo_true_residual(C.byref(self.sys), ptr(dx, C.c_double))

    def solve_coupled(self, h, max_iterations, tolerance, reuse=False, predicted=None):
        pred = None if predicted is None else np.ascontiguousarray(predicted, np.float64).reshape(-1)
        it = C.c_uint32()
        res = C.c_double()
        lib().vxo_solve_coupled(C.byref(self.s), ptr(self.target_mask, C.c_uint8), ptr(self.loads, C.c_double),
                                None if pred is None else ptr(pred, C.c_double), h, max_iterations, tolerance,
                                int(reuse), ptr(self.factor, C.c_double), C.byref(self.sys), C.byref(it),
                                C.byref(res))
        return it.value, res.value

    def bond_stress(self):
        ratio = np.zeros(3 * self.n, np.float64)
        force = np.zeros(9 * self.n, np.float64)
        lib().vxo_bond_stress(C.byref(self.s), C.byref(self.sys), ptr(ratio, C.c_double), ptr(force, C.c_double))
        return ratio.reshape(3, self.n), force.reshape(3, self.n, 3)

    def make_constraint(self, i, axis, j):
        frame, mk, k, rest = np.zeros(9), np.zeros(9), np.zeros(9), np.zeros(3)
        lib().vxo_make_constraint(C.byref(self.s), i, axis, j, ptr(frame, C.c_double), ptr(mk, C.c_double),
                                  ptr(k, C.c_double), ptr(rest, C.c_double))
        return frame.reshape(3, 3), mk.reshape(3, 3), k.reshape(3, 3), rest

    def stiffness_matrix(self, i, j, frame):
        f = np.ascontiguousarray(frame, np.float64).reshape(-1)
        k = np.zeros(9)
        lib().vxo_stiffness_matrix(C.byref(self.s), i, j, ptr(f, C.c_double), ptr(k, C.c_double))
        return k.reshape(3, 3)

    def bond_thermal_rest(self, i, j, frame):
        f = np.ascontiguousarray(frame, np.float64).reshape(-1)
        r = np.zeros(3)
        lib().vxo_bond_thermal_rest(C.byref(self.s), i, j, ptr(f, C.c_double), ptr(r, C.c_double))
        return r

    def bond_limits(self, i, j, direction) -> VxoLimits:
        d = np.ascontiguousarray(direction, np.float64)
        out = VxoLimits()
        lib().vxo_bond_limits(C.byref(self.s), i, j, ptr(d, C.c_double), C.byref(out))
        return out

    def pack_rows(self):
        n = self.n
        active = np.zeros(n, np.uint32)
        rhs = np.zeros(3 * n, np.float32)
        nbr6 = np.zeros(6 * n, np.uint32)
        diag9 = np.zeros(9 * n, np.float32)
        blocks = np.zeros(54 * n, np.float32)
        inv9 = np.zeros(9 * n, np.float32)
        cnt = lib().vxo_pack_rows(C.byref(self.sys), ptr(active, C.c_uint32), ptr(rhs, C.c_float),
                                  ptr(nbr6, C.c_uint32), ptr(diag9, C.c_float), ptr(blocks, C.c_float),
                                  ptr(inv9, C.c_float))
        return dict(active=active[:cnt].copy(), rhs=rhs[:3 * cnt].copy(), nbr6=nbr6[:6 * cnt].copy(),
                    diag9=diag9[:9 * cnt].copy(), blocks54=blocks[:54 * cnt].copy(), inv9=inv9[:9 * cnt].copy(),
                    n=int(cnt))


def basis(axis, q):
    q = np.ascontiguousarray(q, np.float64)
    out = np.zeros(9)
    lib().vxo_basis(axis, ptr(q, C.c_double), ptr(out, C.c_double))
    return out.reshape(3, 3)


def pair_limits(ma, mb, alignment, anisotropy) -> VxoLimits:
    a = material_struct(ma)
    b = material_struct(mb)
    al = np.ascontiguousarray(alignment, np.float64)
    an = np.ascontiguousarray(anisotropy, np.float64)
    out = VxoLimits()
    lib().vxo_pair_limits(C.byref(a), C.byref(b), ptr(al, C.c_double), ptr(an, C.c_double), C.byref(out))
    return out


def fracture_update(bond: VxoBond, u, k, limits: VxoLimits, dt, config: VxoFractureConfig) -> VxoDissipation:
    u = np.ascontiguousarray(u, np.float64)
    k = np.ascontiguousarray(k, np.float64).reshape(-1)
    out = VxoDissipation()
    lib().vxo_fracture_update(C.byref(bond), ptr(u, C.c_double), ptr(k, C.c_double), C.byref(limits), dt,
                              C.byref(config), C.byref(out))
    return out


def fatigue(bond: VxoBond, signed_ratio, config: VxoFractureConfig):
    lib().vxo_fatigue(C.byref(bond), signed_ratio, C.byref(config))


def pcg_rows_f32(rows, max_iterations, tolerance, threads=1):
    n = rows["n"]
    dx = np.zeros(3 * n, np.float32)
    it = C.c_uint32()
    res = C.c_float()
    lib().vxo_pcg_rows_f32(n, ptr(rows["rhs"], C.c_float), ptr(rows["nbr6"], C.c_uint32),
                           ptr(rows["diag9"], C.c_float), ptr(rows["blocks54"], C.c_float), max_iterations,
                           tolerance, threads, ptr(dx, C.c_float), C.byref(it), C.byref(res))
    return dx.reshape(-1, 3), it.value, res.value


def cuda_pcg_emulate(rows, max_iterations, tolerance):
    n = rows["n"]
    dx = np.zeros(3 * max(n, 1), np.float32)
    it = C.c_uint32()
    res = C.c_float()
    st = lib().vxo_cuda_pcg_emulate(n, ptr(rows["rhs"], C.c_float), ptr(rows["nbr6"], C.c_uint32),
                                    ptr(rows["diag9"], C.c_float), ptr(rows["blocks54"], C.c_float),
                                    ptr(rows["inv9"], C.c_float), max_iterations, tolerance,
                                    ptr(dx, C.c_float), C.byref(it), C.byref(res))
    return st, dx[:3 * n].reshape(-1, 3), it.value, res.value


class OracleStepper:
    """vxo_step driver with the dynamic state of solver::step."""

    def __init__(self, scene, *, fixed_dt, substeps, iterations, solver_tolerance=1e-5,
                 corotation_tolerance=1e-5, corotation_iterations=2, gravity=(0, 0, 0),
                 fracture=True, fracture_config=None, contact=False, restitution=0.1, friction=0.35,
                 rest=None):
        self.o = OracleScene(scene)
        n = scene.n
        self.velocity = np.ascontiguousarray(scene.velocity, np.float64).reshape(-1).copy()
        self.previous = self.o.pos.copy()
        self.target = np.ascontiguousarray(scene.target, np.float64).reshape(-1).copy()
        self.bonds = (VxoBond * max(3 * n, 1))()
        for e in range(3 * n):
            b = self.bonds[e]
            b.neighbor = int(self.o.nbr[e])
        self.last_force = np.zeros(9 * max(n, 1), np.float64)
        self.cfg = VxoStepConfig(fixed_dt, substeps, iterations, solver_tolerance, corotation_tolerance,
                                 corotation_iterations, (C.c_double * 3)(*gravity),
                                 fracture_config or default_fracture_config(), int(fracture), int(contact),
                                 restitution, friction)
        # Scene::rest_positions: the creation positions, f32 (src/scene.rs:520-522)
        r = scene.position if rest is None else rest
        self.rest = np.ascontiguousarray(np.asarray(r, np.float32), np.float64).reshape(-1).copy()
        self.d = VxoDynamics(ptr(self.velocity, C.c_double), ptr(self.previous, C.c_double),
                             ptr(self.o.target_mask, C.c_uint8), ptr(self.target, C.c_double),
                             ptr(self.o.loads, C.c_double), self.bonds, ptr(self.last_force, C.c_double),
                             0.0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, ptr(self.rest, C.c_double), 0, 0.0, 0.0)

    def set_targets(self, mask, values):
        self.o.target_mask[:] = mask
        self.target[:] = np.ascontiguousarray(values, np.float64).reshape(-1)

    def step(self):
        lib().vxo_step(C.byref(self.o.s), C.byref(self.cfg), C.byref(self.d))

    @property
    def positions(self):
        return self.o.pos.reshape(-1, 3)

    @property
    def broken(self):
        return self.d.broken

    def last_forces(self):
        return self.last_force.reshape(3, self.o.n, 3)


def rebuild_clusters(neighbor, kinematic):
    """vxo_rebuild_clusters: (clusters[n], cluster_count)."""
    nb = np.ascontiguousarray(neighbor, np.uint32).reshape(-1)
    kin = np.ascontiguousarray(kinematic, np.uint8)
    n = len(kin)
    out = np.zeros(max(n, 1), np.uint32)
    lib().vxo_rebuild_clusters.restype = C.c_uint32
    cnt = lib().vxo_rebuild_clusters(n, ptr(nb, C.c_uint32), ptr(kin, C.c_uint8), ptr(out, C.c_uint32))
    return out[:n].copy(), int(cnt)


def contact_project(position, previous, rest, kinematic, mass, neighbor, target_mask=None):
    """vxo_contact_project (collision::project): corrected (position, previous)
    as (n, 3) arrays, the contacts as a structured array (i, j, normal,
    new_impact) sorted by (i, j), and the pair statistics."""
    pos = np.ascontiguousarray(position, np.float64).reshape(-1).copy()
    prev = np.ascontiguousarray(previous, np.float64).reshape(-1).copy()
    rst = np.ascontiguousarray(np.asarray(rest, np.float32), np.float64).reshape(-1).copy()
    kin = np.ascontiguousarray(kinematic, np.uint8)
    m = np.ascontiguousarray(mass, np.float64)
    nb = np.ascontiguousarray(neighbor, np.uint32).reshape(-1)
    n = len(kin)
    tm = None if target_mask is None else np.ascontiguousarray(target_mask, np.uint8)
    out = C.POINTER(VxoContact)()
    st = VxoContactStats()
    cnt = lib().vxo_contact_project(n, ptr(pos, C.c_double), ptr(prev, C.c_double), ptr(rst, C.c_double),
                                    ptr(kin, C.c_uint8), ptr(m, C.c_double),
                                    None if tm is None else ptr(tm, C.c_uint8), ptr(nb, C.c_uint32),
                                    C.byref(out), C.byref(st))
    contacts = np.zeros(cnt, dtype=CONTACT_DTYPE)
    for k in range(cnt):
        c = out[k]
        contacts[k] = (c.i, c.j, c.normal, c.new_impact)
    lib().free(C.cast(out, C.c_void_p))
    stats = dict(candidates=st.candidates, pairs=st.pairs, contacts=st.contacts, sweeps=st.sweeps)
    return pos.reshape(-1, 3), prev.reshape(-1, 3), contacts, stats


CONTACT_DTYPE = np.dtype([("i", "<u4"), ("j", "<u4"), ("normal", "<i4"), ("new_impact", "<i4")])


def resolve_velocities(velocity, pre_contact, kinematic, mass, contacts, restitution, friction, target_mask=None):
    """vxo_resolve_velocities (resolve_velocities_with_precontact): the new
    (n, 3) velocities and the (restitution, friction) heat."""
    vel = np.ascontiguousarray(velocity, np.float64).reshape(-1).copy()
    pre = np.ascontiguousarray(pre_contact, np.float64).reshape(-1).copy()
    kin = np.ascontiguousarray(kinematic, np.uint8)
    m = np.ascontiguousarray(mass, np.float64)
    tm = None if target_mask is None else np.ascontiguousarray(target_mask, np.uint8)
    arr = (VxoContact * max(len(contacts), 1))()
    for k, c in enumerate(contacts):
        arr[k] = VxoContact(int(c["i"]), int(c["j"]), int(c["normal"]), int(c["new_impact"]), k)
    rh, fh = np.zeros(1), np.zeros(1)
    lib().vxo_resolve_velocities(len(kin), ptr(vel, C.c_double), ptr(pre, C.c_double), ptr(kin, C.c_uint8),
                                 ptr(m, C.c_double), None if tm is None else ptr(tm, C.c_uint8), arr, len(contacts),
                                 restitution, friction, ptr(rh, C.c_double), ptr(fh, C.c_double))
    return vel.reshape(-1, 3), float(rh[0]), float(fh[0])
