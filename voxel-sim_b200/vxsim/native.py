"""ctypes binding of libvxcorot.so (the C ABI declared in include/vxcorot.h).

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np

from . import materials as M

PKG = Path(__file__).resolve().parents[1]
ROOT = PKG.parent
LIB_PATH = PKG / "lib" / "libvxcorot.so"
HEADER = ROOT / "include" / "vxcorot.h"

VX_OK, VX_NOT_CONVERGED, VX_NONFINITE, VX_OOM, VX_BAD_INPUT, VX_CUDA_ERROR, VX_TIMEOUT, VX_NO_DEVICE = range(8)
PRECISION_FP64, PRECISION_MIXED = 0, 1
KERNEL_AUTO, KERNEL_STREAMING, KERNEL_PERSISTENT = 0, 1, 2
EMPTY = 0xFFFFFFFF

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)


class VxError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"status {status}: {message}")
        self.status = status


class VxMaterial(C.Structure):
    _fields_ = [(name, C.c_float) for name in M.MATERIAL_DTYPE.names[:-1]] + [("fracture_mode", C.c_int32)]


class VxSceneDesc(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("position", f64p), ("rotation", f64p), ("kinematic", u8p), ("mass", f32p),
        ("material", u32p), ("materials", C.POINTER(VxMaterial)), ("material_count", C.c_uint32),
        ("fiber", f32p), ("anisotropy", f32p), ("solid_fraction", f32p), ("thermal_strength", f32p),
        ("thermal_delta", f32p), ("neighbor", u32p), ("formation_offset", f32p), ("plastic_strain", f32p),
        ("damage", f32p),
    ]


class VxPassParams(C.Structure):
    _fields_ = [("h", C.c_double), ("tolerance", C.c_double), ("max_iterations", C.c_uint32),
                ("precision", C.c_int32), ("reuse_preconditioner", C.c_int32), ("inner_tolerance", C.c_double),
                ("max_outer", C.c_uint32), ("kernel", C.c_int32)]


class VxPassStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("outer_iterations", C.c_uint32), ("residual", C.c_double),
                ("true_residual", C.c_double), ("active", C.c_uint32), ("bonds_assembled", C.c_uint32),
                ("converged", C.c_int32), ("kernel_launches", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VxFractureConfig(C.Structure):
    _fields_ = [("damage_rate", C.c_double), ("energy_release", C.c_double), ("fatigue_cycles", C.c_double),
                ("fatigue_exponent", C.c_double), ("fatigue_threshold", C.c_double),
                ("plastic_heat_fraction", C.c_double)]


def fracture_config(damage_rate=35.0, energy_release=0.005, fatigue_cycles=1000.0, fatigue_exponent=3.0,
                    fatigue_threshold=0.5, plastic_heat_fraction=0.9) -> VxFractureConfig:
    """FractureConfig::default (src/fracture.rs:27-42)."""
    return VxFractureConfig(damage_rate, energy_release, fatigue_cycles, fatigue_exponent, fatigue_threshold,
                            plastic_heat_fraction)


class VxDissipation(C.Structure):
    _fields_ = [("plastic_heat", C.c_double), ("stored_plastic", C.c_double), ("surface_work", C.c_double),
                ("damage_heat", C.c_double), ("released", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VxStepParams(C.Structure):
    _fields_ = [("fixed_dt", C.c_double), ("substeps", C.c_uint32), ("corotation_iterations", C.c_uint32),
                ("corotation_tolerance", C.c_double), ("gravity", C.c_double * 3), ("pass_", VxPassParams),
                ("fracture", C.c_int32), ("fracture_config", VxFractureConfig), ("contact", C.c_int32),
                ("restitution", C.c_double), ("friction", C.c_double)]


class VxStepStats(C.Structure):
    _fields_ = [("passes", C.c_uint32), ("pcg_iterations", C.c_uint32), ("residual", C.c_double),
                ("max_angle", C.c_double), ("converged", C.c_int32), ("broken", C.c_uint32),
                ("dissipation", VxDissipation), ("contacts", C.c_uint32), ("restitution_heat", C.c_double),
                ("friction_heat", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["dissipation"] = self.dissipation.as_dict()
        return d


class VxContactStats(C.Structure):
    _fields_ = [("candidates", C.c_uint64), ("pairs", C.c_uint64), ("contacts", C.c_uint32), ("sweeps", C.c_uint32),
                ("live_max", C.c_uint32), ("redone", C.c_uint32), ("launches", C.c_uint32), ("stored", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VxContactHeat(C.Structure):
    _fields_ = [("restitution", C.c_double), ("friction", C.c_double)]


FIELD_POSITION, FIELD_VELOCITY, FIELD_PREVIOUS = 0, 1, 2


PERSIST_FORMS = {1: "brick, 1 thread/REV, >=256 REVs/block", 2: "brick, 2 threads/REV, >=256 REVs/block",
                 3: "brick, 1 thread/REV, >=128 REVs/block", 4: "brick, 2 threads/REV, >=128 REVs/block",
                 5: "range (classic recurrence)", 6: "range (one reduction per iteration)",
                 7: "range (classic recurrence), 608 threads/block", 8: "range (classic recurrence), 768 threads/block",
                 9: "range (classic recurrence), 896 threads/block"}


# threads per block of the range-plan forms (VX_PERSIST_RANGE, _608, _768, _896)
RANGE_THREADS = {5: 512, 7: 608, 8: 768, 9: 896}


def tune_label(kernel: int, blocks: int) -> str:
    """Readable name of an autotuner candidate (kernel, blocks field)."""
    if kernel == KERNEL_PERSISTENT:
        return "persistent " + PERSIST_FORMS.get(blocks, str(blocks))
    return f"streaming, {blocks} blocks/SM"


class VxTuneResult(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("blocks_per_sm", C.c_int32), ("us_per_iteration", C.c_double),
                ("from_cache", C.c_int32), ("candidates", C.c_uint32), ("candidate_kernel", C.c_int32 * 12),
                ("candidate_blocks", C.c_int32 * 12), ("candidate_us", C.c_double * 12)]

    def as_dict(self):
        k = self.candidates
        return {"kernel": self.kernel, "blocks_per_sm": self.blocks_per_sm,
                "us_per_iteration": self.us_per_iteration, "from_cache": self.from_cache,
                "candidates": [(self.candidate_kernel[i], self.candidate_blocks[i], self.candidate_us[i])
                               for i in range(k)]}


class VxServerConfig(C.Structure):
    _fields_ = [("max_revs", C.c_uint64), ("hbm_fraction", C.c_double), ("max_slots", C.c_uint32),
                ("step", VxStepParams), ("lanes", C.c_uint32), ("lane_max_revs", C.c_uint32 * 3)]


class VxRequestPlan(C.Structure):
    _fields_ = [("steps", C.c_uint32), ("target_velocity", C.c_double * 3)]


class VxRequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("n", C.c_uint32), ("steps_done", C.c_uint32), ("passes", C.c_uint32),
                ("pcg_iterations", C.c_uint64), ("worst_residual", C.c_double), ("queued_s", C.c_double),
                ("run_s", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VxServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("resident", C.c_uint32), ("queued", C.c_uint32), ("rounds", C.c_uint64),
                ("scene_steps", C.c_uint64), ("solves", C.c_uint64), ("elapsed_s", C.c_double),
                ("busy_s", C.c_double), ("p50_step_ms", C.c_double), ("p99_step_ms", C.c_double),
                ("max_step_ms", C.c_double), ("pool_revs", C.c_uint64), ("pool_bytes", C.c_uint64),
                ("worst_residual", C.c_double), ("not_converged", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def step_params(fixed_dt, substeps=1, corotation_iterations=2, corotation_tolerance=1e-5, gravity=(0.0, 0.0, 0.0),
                tolerance=1e-5, max_iterations=10000, precision=PRECISION_FP64, reuse=False, inner_tolerance=0.0,
                max_outer=0, kernel=KERNEL_AUTO, fracture=False, fracture_cfg=None, contact=False,
                restitution=0.1, friction=0.35) -> VxStepParams:
    return VxStepParams(fixed_dt, substeps, corotation_iterations, corotation_tolerance, (C.c_double * 3)(*gravity),
                        VxPassParams(fixed_dt / substeps, tolerance, max_iterations, precision, int(reuse),
                                     inner_tolerance, max_outer, kernel),
                        int(fracture), fracture_cfg or fracture_config(), int(contact), restitution, friction)


_lib = None


def header_symbols() -> list[str]:
    """Function names declared in include/vxcorot.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vx_[a-z0-9_]+)\s*\(", text)))


def load(path: Path | None = None):
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("VXCOROT_LIB", LIB_PATH))
    if not p.exists():
        raise RuntimeError(f"libvxcorot.so not built at {p}; run __graft_entry__.build() or make -C voxel-sim_b200")
    L = C.CDLL(str(p))
    L.vx_last_error.restype = C.c_char_p
    L.vx_abi_version.restype = C.c_int32
    L.vx_ctx_create.argtypes = [C.c_int32, C.POINTER(C.c_void_p)]
    L.vx_ctx_destroy.argtypes = [C.c_void_p]
    L.vx_build_topology.argtypes = [C.c_void_p, i32p, u8p, C.c_uint32, u32p]
    L.vx_scene_create.argtypes = [C.c_void_p, C.POINTER(VxSceneDesc), C.POINTER(C.c_void_p)]
    L.vx_scene_destroy.argtypes = [C.c_void_p]
    L.vx_scene_footprint_bytes.restype = C.c_uint64
    L.vx_scene_footprint_bytes.argtypes = [C.c_uint32]
    for name in ("vx_scene_set_positions", "vx_scene_get_positions", "vx_scene_set_rotations",
                 "vx_scene_get_rotations", "vx_scene_set_loads", "vx_scene_set_predicted",
                 "vx_scene_set_previous"):
        getattr(L, name).argtypes = [C.c_void_p, f64p]
    L.vx_scene_set_targets.argtypes = [C.c_void_p, u8p, f64p]
    L.vx_scene_set_bonds.argtypes = [C.c_void_p, u32p, f32p, f32p, f32p]
    L.vx_scene_get_neighbors.argtypes = [C.c_void_p, u32p]
    L.vx_fit_rotations.argtypes = [C.c_void_p, f64p]
    L.vx_corotational_pass.argtypes = [C.c_void_p, C.POINTER(VxPassParams), C.POINTER(VxPassStats)]
    L.vx_bond_stress.argtypes = [C.c_void_p, f32p, f32p, u32p, C.c_uint32, u32p]
    L.vx_solve_pcg_f32.argtypes = [f32p, u32p, f32p, f32p, f32p, C.c_uint32, C.c_uint32, C.c_float, f32p, u32p, f32p]
    L.vx_solve_pcg_f32_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_uint32, C.c_float, C.c_void_p, u32p, f32p, C.c_void_p]
    L.vx_scene_checkpoint.argtypes = [C.c_void_p, C.c_int32]
    L.vx_scene_stream.restype = C.c_void_p
    L.vx_scene_stream.argtypes = [C.c_void_p]
    L.vx_scene_kernel_times.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_void_p, C.c_uint64, f64p]
    L.vx_scene_step.argtypes = [C.c_void_p, C.POINTER(VxStepParams), C.POINTER(VxStepStats)]
    L.vx_fracture_commit.argtypes = [C.c_void_p, C.c_double, C.POINTER(VxFractureConfig), C.POINTER(VxDissipation),
                                     C.POINTER(C.c_uint32)]
    L.vx_scene_get_bond_state.argtypes = [C.c_void_p, f32p, f32p, f32p, f32p]
    L.vx_scene_get_last_forces.argtypes = [C.c_void_p, f32p]
    L.vx_scene_rebuild_clusters.argtypes = [C.c_void_p, u32p, C.POINTER(C.c_uint32)]
    L.vx_scene_autotune.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.POINTER(VxTuneResult)]
    L.vx_server_create.argtypes = [C.c_void_p, C.POINTER(VxServerConfig), C.POINTER(C.c_void_p)]
    L.vx_server_submit.argtypes = [C.c_void_p, C.POINTER(VxSceneDesc), u8p, f64p, C.POINTER(VxRequestPlan),
                                   C.POINTER(C.c_uint64)]
    L.vx_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(VxRequestResult), f64p]
    L.vx_server_get_stats.argtypes = [C.c_void_p, C.POINTER(VxServerStats)]
    L.vx_server_destroy.argtypes = [C.c_void_p]
    L.vx_scene_set_velocities.argtypes = [C.c_void_p, f64p]
    L.vx_scene_get_velocities.argtypes = [C.c_void_p, f64p]
    L.vx_scene_update_velocities.argtypes = [C.c_void_p, C.c_uint32, u32p, f64p, C.c_int32]
    L.vx_scene_read_revs.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, u32p, f64p]
    L.vx_scene_write_revs.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, u32p, f64p]
    L.vx_contact_project.argtypes = [C.c_void_p, C.POINTER(VxContactStats)]
    L.vx_contact_resolve_velocities.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double,
                                                C.POINTER(VxContactHeat)]
    L.vx_scene_get_contacts.argtypes = [C.c_void_p, C.c_uint32, u32p, u32p, i32p, u8p, C.POINTER(C.c_uint32)]
    L.vx_scene_set_contacts.argtypes = [C.c_void_p, C.c_uint32, u32p, u32p, i32p, u8p]
    for name in header_symbols():
        getattr(L, name)  # every declared entry point is exported
    _lib = L
    return L


def last_error() -> str:
    return load().vx_last_error().decode()


def check(status, allow=()):
    if status != VX_OK and status not in allow:
        raise VxError(status, last_error())
    return status


def _p(a, ct):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ct))


class Context:
    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(load().vx_ctx_create(device, C.byref(self.h)))

    def close(self):
        if self.h:
            load().vx_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build_topology(self, cells, kinematic) -> np.ndarray:
        cells = np.ascontiguousarray(cells, np.int32).reshape(-1, 3)
        kin = np.ascontiguousarray(kinematic, np.uint8)
        out = np.zeros(3 * len(cells), np.uint32)
        check(load().vx_build_topology(self.h, _p(cells, C.c_int32), _p(kin, C.c_uint8), len(cells),
                                       _p(out, C.c_uint32)))
        return out.reshape(3, -1)


def material_array(materials):
    arr = (VxMaterial * max(len(materials), 1))()
    for k, m in enumerate(materials):
        for name, _ in VxMaterial._fields_:
            setattr(arr[k], name, getattr(m, name))
    return arr


class DeviceScene:
    """A scene resident on the device (vx_scene handle)."""

    def __init__(self, ctx: Context, scene):
        self.ctx = ctx
        self.n = scene.n
        self._keep = dict(
            pos=np.ascontiguousarray(scene.position, np.float64).reshape(-1),
            rot=np.ascontiguousarray(scene.rotation, np.float64).reshape(-1),
            kin=np.ascontiguousarray(scene.kinematic, np.uint8),
            mass=np.ascontiguousarray(scene.mass, np.float32),
            mat=np.ascontiguousarray(scene.material, np.uint32),
            fib=np.ascontiguousarray(scene.fiber, np.float32).reshape(-1),
            ani=np.ascontiguousarray(scene.anisotropy, np.float32),
            solid=np.ascontiguousarray(scene.solid_fraction, np.float32),
            therm=np.ascontiguousarray(scene.thermal_strength, np.float32),
            dT=np.ascontiguousarray(scene.thermal_delta, np.float32),
            nbr=np.ascontiguousarray(scene.neighbor, np.uint32).reshape(-1),
            form=np.ascontiguousarray(scene.formation_offset, np.float32).reshape(-1),
            plas=np.ascontiguousarray(scene.plastic_strain, np.float32).reshape(-1),
            dmg=np.ascontiguousarray(scene.damage, np.float32).reshape(-1),
        )
        k = self._keep
        self._mats = material_array(scene.materials)
        desc = VxSceneDesc(
            scene.n, _p(k["pos"], C.c_double), _p(k["rot"], C.c_double), _p(k["kin"], C.c_uint8),
            _p(k["mass"], C.c_float), _p(k["mat"], C.c_uint32), self._mats, len(scene.materials),
            _p(k["fib"], C.c_float), _p(k["ani"], C.c_float), _p(k["solid"], C.c_float),
            _p(k["therm"], C.c_float), _p(k["dT"], C.c_float), _p(k["nbr"], C.c_uint32),
            _p(k["form"], C.c_float), _p(k["plas"], C.c_float), _p(k["dmg"], C.c_float))
        self.h = C.c_void_p()
        check(load().vx_scene_create(ctx.h, C.byref(desc), C.byref(self.h)))
        self.set_targets(scene.target_mask, scene.target)
        self.set_loads(scene.loads)

    def close(self):
        if self.h:
            load().vx_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ----------------------------------------------------------------
    def _vec(self, a):
        return np.ascontiguousarray(a, np.float64).reshape(-1)

    def set_positions(self, x):
        x = self._vec(x)
        check(load().vx_scene_set_positions(self.h, _p(x, C.c_double)))

    def set_previous(self, xyz):
        """Previous positions (the contact projection's swept starts) of every REV."""
        x = self._vec(xyz)
        check(load().vx_scene_set_previous(self.h, _p(x, C.c_double)))

    def positions(self, out=None) -> np.ndarray:
        """Positions (n, 3); `out` (a C-contiguous float64 array of 3n values,
        pinned for a direct copy) receives them when given."""
        out = np.zeros(3 * self.n, np.float64) if out is None else out
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.size == 3 * self.n
        check(load().vx_scene_get_positions(self.h, _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def set_rotations(self, q):
        q = self._vec(q)
        check(load().vx_scene_set_rotations(self.h, _p(q, C.c_double)))

    def rotations(self) -> np.ndarray:
        out = np.zeros(4 * self.n, np.float64)
        check(load().vx_scene_get_rotations(self.h, _p(out, C.c_double)))
        return out.reshape(-1, 4)

    def set_targets(self, mask, target=None):
        mask = np.ascontiguousarray(mask, np.uint8)
        t = None if target is None else self._vec(target)
        check(load().vx_scene_set_targets(self.h, _p(mask, C.c_uint8), _p(t, C.c_double)))

    def set_loads(self, loads):
        x = self._vec(loads)
        check(load().vx_scene_set_loads(self.h, _p(x, C.c_double)))

    def set_predicted(self, x=None):
        x = None if x is None else self._vec(x)
        check(load().vx_scene_set_predicted(self.h, _p(x, C.c_double)))

    def set_bonds(self, neighbor, plastic=None, damage=None, formation=None):
        nb = np.ascontiguousarray(neighbor, np.uint32).reshape(-1)
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1)
        pl, dm, fo = f(plastic), f(damage), f(formation)
        check(load().vx_scene_set_bonds(self.h, _p(nb, C.c_uint32), _p(pl, C.c_float), _p(dm, C.c_float),
                                        _p(fo, C.c_float)))

    def neighbors(self) -> np.ndarray:
        out = np.zeros(3 * self.n, np.uint32)
        check(load().vx_scene_get_neighbors(self.h, _p(out, C.c_uint32)))
        return out.reshape(3, -1)

    def save_state(self):
        check(load().vx_scene_checkpoint(self.h, 0))

    def restore_state(self):
        check(load().vx_scene_checkpoint(self.h, 1))

    @property
    def stream_ptr(self) -> int:
        return int(load().vx_scene_stream(self.h) or 0)

    def kernel_times(self, precision, reps=20, flush_ptr=0, flush_bytes=0):
        out = np.zeros(5, np.float64)
        check(load().vx_scene_kernel_times(self.h, precision, reps, C.c_void_p(flush_ptr), flush_bytes,
                                           _p(out, C.c_double)))
        return {"matvec_us": float(out[0]), "update_us": float(out[1]), "persistent_iter_us": float(out[2]),
                "persistent_iterations": int(out[3]),
                "persistent_form": {0: None, 1: "brick", 2: "range", 3: "expanded"}[int(out[4])]}

    # -- the solve ------------------------------------------------------------
    def fit_rotations(self) -> float:
        v = C.c_double()
        check(load().vx_fit_rotations(self.h, C.byref(v)))
        return v.value

    def corotational_pass(self, h, tolerance, max_iterations, precision=PRECISION_FP64, reuse=False,
                          inner_tolerance=0.0, max_outer=0, kernel=KERNEL_AUTO, allow=(VX_NOT_CONVERGED,)):
        p = VxPassParams(h, tolerance, max_iterations, precision, int(reuse), inner_tolerance, max_outer, kernel)
        st = VxPassStats()
        status = check(load().vx_corotational_pass(self.h, C.byref(p), C.byref(st)), allow=allow)
        d = st.as_dict()
        d["status"] = status
        return d

    def step(self, params: VxStepParams, allow=(VX_NOT_CONVERGED,)):
        st = VxStepStats()
        status = check(load().vx_scene_step(self.h, C.byref(params), C.byref(st)), allow=allow)
        d = st.as_dict()
        d["status"] = status
        return d

    def fracture_commit(self, dt, cfg=None):
        d, broken = VxDissipation(), C.c_uint32()
        check(load().vx_fracture_commit(self.h, dt, C.byref(cfg or fracture_config()), C.byref(d), C.byref(broken)))
        return d.as_dict(), broken.value

    def autotune(self, precision=PRECISION_MIXED, cache_path=None) -> dict:
        """vx_scene_autotune: times the candidate launch configurations of the
        inner solve (after a pass) and keeps the fastest for later passes."""
        out = VxTuneResult()
        path = None if cache_path is None else str(cache_path).encode()
        check(load().vx_scene_autotune(self.h, precision, path, C.byref(out)))
        return out.as_dict()

    def rebuild_clusters(self):
        """(clusters[n], cluster_count) as rebuild_clusters numbers them."""
        out = np.zeros(max(self.n, 1), np.uint32)
        cnt = C.c_uint32()
        check(load().vx_scene_rebuild_clusters(self.h, _p(out, C.c_uint32), C.byref(cnt)))
        return out[:self.n].copy(), cnt.value

    def bond_state(self):
        m = 3 * self.n
        pl, dm, ep, fa = (np.zeros(3 * m, np.float32), np.zeros(m, np.float32), np.zeros(m, np.float32),
                          np.zeros(m, np.float32))
        check(load().vx_scene_get_bond_state(self.h, _p(pl, C.c_float), _p(dm, C.c_float), _p(ep, C.c_float),
                                             _p(fa, C.c_float)))
        return dict(plastic=pl.reshape(3, -1, 3), damage=dm.reshape(3, -1), eq_plastic=ep.reshape(3, -1),
                    fatigue=fa.reshape(3, -1))

    def last_forces(self) -> np.ndarray:
        """Bond workspace last_force of the last fracture commit, (3, n, 3) f32 N."""
        out = np.zeros(9 * self.n, np.float32)
        check(load().vx_scene_get_last_forces(self.h, _p(out, C.c_float)))
        return out.reshape(3, -1, 3)

    def set_velocities(self, v):
        v = self._vec(v)
        check(load().vx_scene_set_velocities(self.h, _p(v, C.c_double)))

    def velocities(self) -> np.ndarray:
        out = np.zeros(3 * self.n, np.float64)
        check(load().vx_scene_get_velocities(self.h, _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def write_field(self, field, values, index=None):
        """vx_scene_write_revs: every REV (index None) or the listed ones."""
        idx = np.arange(self.n, dtype=np.uint32) if index is None else np.ascontiguousarray(index, np.uint32)
        val = np.ascontiguousarray(values, np.float64).reshape(-1)
        check(load().vx_scene_write_revs(self.h, field, len(idx), _p(idx, C.c_uint32), _p(val, C.c_double)))

    def read_field(self, field, index=None) -> np.ndarray:
        idx = np.arange(self.n, dtype=np.uint32) if index is None else np.ascontiguousarray(index, np.uint32)
        out = np.zeros(3 * len(idx), np.float64)
        check(load().vx_scene_read_revs(self.h, field, len(idx), _p(idx, C.c_uint32), _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def contact_project(self) -> dict:
        """vx_contact_project (collision::project) over the current positions,
        with the previous positions as the swept starts."""
        st = VxContactStats()
        check(load().vx_contact_project(self.h, C.byref(st)))
        return st.as_dict()

    def contacts(self) -> np.ndarray:
        """The current contacts as a structured array (i, j, normal, new_impact)."""
        cnt = C.c_uint32()
        check(load().vx_scene_get_contacts(self.h, 0, None, None, None, None, C.byref(cnt)))
        k = cnt.value
        i, j, nrm, imp = (np.zeros(max(k, 1), np.uint32), np.zeros(max(k, 1), np.uint32),
                          np.zeros(max(k, 1), np.int32), np.zeros(max(k, 1), np.uint8))
        if k:
            check(load().vx_scene_get_contacts(self.h, k, _p(i, C.c_uint32), _p(j, C.c_uint32), _p(nrm, C.c_int32),
                                               _p(imp, C.c_uint8), C.byref(cnt)))
        out = np.zeros(k, dtype=[("i", "<u4"), ("j", "<u4"), ("normal", "<i4"), ("new_impact", "<i4")])
        out["i"], out["j"], out["normal"], out["new_impact"] = i[:k], j[:k], nrm[:k], imp[:k]
        return out

    def set_contacts(self, contacts):
        c = np.asarray(contacts)
        i = np.ascontiguousarray(c["i"], np.uint32)
        j = np.ascontiguousarray(c["j"], np.uint32)
        nrm = np.ascontiguousarray(c["normal"], np.int32)
        imp = np.ascontiguousarray(c["new_impact"], np.uint8)
        check(load().vx_scene_set_contacts(self.h, len(i), _p(i, C.c_uint32), _p(j, C.c_uint32),
                                           _p(nrm, C.c_int32), _p(imp, C.c_uint8)))

    def resolve_contact_velocities(self, restitution, friction, pre_contact=0):
        heat = VxContactHeat()
        check(load().vx_contact_resolve_velocities(self.h, pre_contact, restitution, friction, C.byref(heat)))
        return heat.restitution, heat.friction

    def update_velocities(self, index, values, add=False):
        idx = np.ascontiguousarray(index, np.uint32).reshape(-1)
        val = np.ascontiguousarray(values, np.float64).reshape(-1)
        check(load().vx_scene_update_velocities(self.h, len(idx), _p(idx, C.c_uint32), _p(val, C.c_double),
                                                1 if add else 0))

    def bond_stress(self, with_force=True, with_ratio=True, cap=None, ratio_out=None):
        m = 3 * self.n
        ratio = (np.zeros(m, np.float32) if ratio_out is None else ratio_out) if with_ratio else None
        force = np.zeros(3 * m, np.float32) if with_force else None
        cap = m if cap is None else cap
        near = np.zeros(max(cap, 1), np.uint32)
        cnt = C.c_uint32()
        check(load().vx_bond_stress(self.h, _p(ratio, C.c_float), _p(force, C.c_float), _p(near, C.c_uint32), cap,
                                    C.byref(cnt)))
        out = dict(near=near[:min(cnt.value, cap)].copy(), near_count=cnt.value)
        if with_ratio:
            out["ratio"] = ratio.reshape(3, -1)
        if with_force:
            out["force"] = force.reshape(3, -1, 3)
        return out


def solve_pcg_f32(rows, max_iterations, tolerance):
    """vx_solve_pcg_f32 on a packed active-row system (dict of flat arrays)."""
    n = rows["n"]
    dx = np.zeros(3 * max(n, 1), np.float32)
    it = C.c_uint32()
    rel = C.c_float()
    a = {k: np.ascontiguousarray(rows[k]) for k in ("rhs", "nbr6", "diag9", "blocks54", "inv9")}
    st = load().vx_solve_pcg_f32(_p(a["rhs"], C.c_float), _p(a["nbr6"], C.c_uint32), _p(a["diag9"], C.c_float),
                                 _p(a["blocks54"], C.c_float), _p(a["inv9"], C.c_float), n, max_iterations,
                                 tolerance, _p(dx, C.c_float), C.byref(it), C.byref(rel))
    return st, dx[:3 * n].reshape(-1, 3), it.value, rel.value


def scene_desc(scene, keep: dict):
    """vx_scene_desc for a vxsim Scene; `keep` holds the arrays alive."""
    keep.update(
        pos=np.ascontiguousarray(scene.position, np.float64).reshape(-1),
        rot=np.ascontiguousarray(scene.rotation, np.float64).reshape(-1),
        kin=np.ascontiguousarray(scene.kinematic, np.uint8),
        mass=np.ascontiguousarray(scene.mass, np.float32),
        mat=np.ascontiguousarray(scene.material, np.uint32),
        fib=np.ascontiguousarray(scene.fiber, np.float32).reshape(-1),
        ani=np.ascontiguousarray(scene.anisotropy, np.float32),
        solid=np.ascontiguousarray(scene.solid_fraction, np.float32),
        therm=np.ascontiguousarray(scene.thermal_strength, np.float32),
        dT=np.ascontiguousarray(scene.thermal_delta, np.float32),
        nbr=np.ascontiguousarray(scene.neighbor, np.uint32).reshape(-1),
        form=np.ascontiguousarray(scene.formation_offset, np.float32).reshape(-1),
        plas=np.ascontiguousarray(scene.plastic_strain, np.float32).reshape(-1),
        dmg=np.ascontiguousarray(scene.damage, np.float32).reshape(-1),
        mats=material_array(scene.materials),
    )
    k = keep
    return VxSceneDesc(
        scene.n, _p(k["pos"], C.c_double), _p(k["rot"], C.c_double), _p(k["kin"], C.c_uint8),
        _p(k["mass"], C.c_float), _p(k["mat"], C.c_uint32), k["mats"], len(scene.materials),
        _p(k["fib"], C.c_float), _p(k["ani"], C.c_float), _p(k["solid"], C.c_float), _p(k["therm"], C.c_float),
        _p(k["dT"], C.c_float), _p(k["nbr"], C.c_uint32), _p(k["form"], C.c_float), _p(k["plas"], C.c_float),
        _p(k["dmg"], C.c_float))


def _bind_pool(L):
    L.vx_pool_create.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p)]
    L.vx_pool_destroy.argtypes = [C.c_void_p]
    L.vx_pool_footprint_bytes.restype = C.c_uint64
    L.vx_pool_footprint_bytes.argtypes = [C.c_uint64, C.c_uint32]
    L.vx_pool_capacity_slots.restype = C.c_uint32
    L.vx_pool_capacity_slots.argtypes = [C.c_void_p]
    L.vx_pool_free_revs.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.vx_pool_add.argtypes = [C.c_void_p, C.POINTER(VxSceneDesc), C.POINTER(C.c_uint32)]
    L.vx_pool_remove.argtypes = [C.c_void_p, C.c_uint32]
    for name in ("vx_pool_set_positions", "vx_pool_get_positions", "vx_pool_get_rotations", "vx_pool_set_loads",
                 "vx_pool_set_predicted", "vx_pool_set_velocities", "vx_pool_get_velocities",
                 "vx_pool_set_previous", "vx_pool_get_previous"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_uint32, f64p]
    L.vx_pool_set_targets.argtypes = [C.c_void_p, C.c_uint32, u8p, f64p]
    L.vx_pool_advance_targets.argtypes = [C.c_void_p, u8p, f64p]
    L.vx_pool_fit_rotations.argtypes = [C.c_void_p, u8p, f64p]
    L.vx_pool_pass.argtypes = [C.c_void_p, u8p, C.POINTER(VxPassParams), C.POINTER(VxPassStats)]
    L.vx_pool_bond_stress.argtypes = [C.c_void_p, C.c_uint32, f32p, f32p, u32p, C.c_uint32, u32p]
    L.vx_pool_step.argtypes = [C.c_void_p, u8p, C.POINTER(VxStepParams), C.POINTER(VxStepStats)]
    L.vx_pool_contact_project.argtypes = [C.c_void_p, u8p, C.POINTER(VxContactStats), u32p]
    L.vx_pool_checkpoint.argtypes = [C.c_void_p, C.c_int32]
    L.vx_pool_stream.restype = C.c_void_p
    L.vx_pool_stream.argtypes = [C.c_void_p]


class DevicePool:
    """Scenes resident in one device arena (vx_pool), solved together."""

    def __init__(self, ctx: Context, max_revs: int, max_slots: int):
        L = load()
        if not getattr(L, "_pool_bound", False):
            _bind_pool(L)
            L._pool_bound = True
        self.ctx = ctx
        self.h = C.c_void_p()
        check(L.vx_pool_create(ctx.h, max_revs, max_slots, C.byref(self.h)))
        self.slots = max_slots
        self.n = {}

    def close(self):
        if self.h:
            load().vx_pool_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, scene) -> int:
        keep = {}
        desc = scene_desc(scene, keep)
        slot = C.c_uint32()
        check(load().vx_pool_add(self.h, C.byref(desc), C.byref(slot)))
        s = slot.value
        self.n[s] = scene.n
        self.set_targets(s, scene.target_mask, scene.target)
        if np.any(scene.loads):
            self.set_loads(s, scene.loads)
        return s

    def remove(self, slot):
        check(load().vx_pool_remove(self.h, slot))
        self.n.pop(slot, None)

    def free_revs(self):
        a, b = C.c_uint64(), C.c_uint64()
        check(load().vx_pool_free_revs(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def _v(self, a):
        return np.ascontiguousarray(a, np.float64).reshape(-1)

    def set_positions(self, slot, x):
        x = self._v(x)
        check(load().vx_pool_set_positions(self.h, slot, _p(x, C.c_double)))

    def positions(self, slot):
        out = np.zeros(3 * self.n[slot], np.float64)
        check(load().vx_pool_get_positions(self.h, slot, _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def rotations(self, slot):
        out = np.zeros(4 * self.n[slot], np.float64)
        check(load().vx_pool_get_rotations(self.h, slot, _p(out, C.c_double)))
        return out.reshape(-1, 4)

    def advance_targets(self, delta, enabled=None):
        """Moves the targets marked VX_TARGET_MOVING of every selected slot by
        delta[slot] (slots x 3 metres)."""
        m = self._mask(enabled)
        d = np.ascontiguousarray(delta, np.float64).reshape(-1)
        check(load().vx_pool_advance_targets(self.h, _p(m, C.c_uint8), _p(d, C.c_double)))

    def set_targets(self, slot, mask, target=None):
        m = np.ascontiguousarray(mask, np.uint8)
        t = None if target is None else self._v(target)
        check(load().vx_pool_set_targets(self.h, slot, _p(m, C.c_uint8), _p(t, C.c_double)))

    def set_loads(self, slot, loads):
        x = self._v(loads)
        check(load().vx_pool_set_loads(self.h, slot, _p(x, C.c_double)))

    def set_predicted(self, slot, x=None):
        x = None if x is None else self._v(x)
        check(load().vx_pool_set_predicted(self.h, slot, _p(x, C.c_double)))

    def set_velocities(self, slot, v):
        x = self._v(v)
        check(load().vx_pool_set_velocities(self.h, slot, _p(x, C.c_double)))

    def set_previous(self, slot, x):
        x = self._v(x)
        check(load().vx_pool_set_previous(self.h, slot, _p(x, C.c_double)))

    def previous(self, slot):
        out = np.zeros(3 * self.n[slot], np.float64)
        check(load().vx_pool_get_previous(self.h, slot, _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def contact_project(self, enabled=None):
        """vx_pool_contact_project: (call statistics, contacts per slot)."""
        m = self._mask(enabled)
        st = VxContactStats()
        per = np.zeros(self.slots, np.uint32)
        check(load().vx_pool_contact_project(self.h, _p(m, C.c_uint8), C.byref(st), _p(per, C.c_uint32)))
        return st.as_dict(), per

    def velocities(self, slot) -> np.ndarray:
        out = np.zeros(3 * self.n[slot], np.float64)
        check(load().vx_pool_get_velocities(self.h, slot, _p(out, C.c_double)))
        return out.reshape(-1, 3)

    def step(self, params: "VxStepParams", enabled=None, allow=(VX_NOT_CONVERGED,)):
        """vx_pool_step: one fixed step of every selected slot; per-slot stats."""
        m = self._mask(enabled)
        stats = (VxStepStats * self.slots)()
        status = check(load().vx_pool_step(self.h, _p(m, C.c_uint8), C.byref(params), stats), allow=allow)
        return status, [stats[k].as_dict() for k in range(self.slots)]

    def _mask(self, enabled):
        if enabled is None:
            return None
        m = np.zeros(self.slots, np.uint8)
        m[list(enabled)] = 1
        return m

    def fit_rotations(self, enabled=None):
        m = self._mask(enabled)
        out = np.zeros(self.slots, np.float64)
        check(load().vx_pool_fit_rotations(self.h, _p(m, C.c_uint8), _p(out, C.c_double)))
        return out

    def corotational_pass(self, h, tolerance, max_iterations, enabled=None, reuse=False, inner_tolerance=0.0,
                          max_outer=0, kernel=KERNEL_AUTO, allow=(VX_NOT_CONVERGED,)):
        """One pass of every selected slot. kernel: KERNEL_PERSISTENT solves the
        slots in waves of the persistent kernel, KERNEL_AUTO / KERNEL_STREAMING
        with the tile kernels."""
        m = self._mask(enabled)
        p = VxPassParams(h, tolerance, max_iterations, PRECISION_MIXED, int(reuse), inner_tolerance, max_outer,
                         kernel)
        stats = (VxPassStats * self.slots)()
        status = check(load().vx_pool_pass(self.h, _p(m, C.c_uint8), C.byref(p), stats), allow=allow)
        return status, [stats[k].as_dict() for k in range(self.slots)]

    def bond_stress(self, slot, with_force=True):
        n = self.n[slot]
        ratio = np.zeros(3 * n, np.float32)
        force = np.zeros(9 * n, np.float32) if with_force else None
        near = np.zeros(3 * n, np.uint32)
        cnt = C.c_uint32()
        check(load().vx_pool_bond_stress(self.h, slot, _p(ratio, C.c_float), _p(force, C.c_float),
                                         _p(near, C.c_uint32), 3 * n, C.byref(cnt)))
        out = dict(ratio=ratio.reshape(3, -1), near=near[:cnt.value].copy())
        if with_force:
            out["force"] = force.reshape(3, -1, 3)
        return out

    def save_state(self):
        check(load().vx_pool_checkpoint(self.h, 0))

    def restore_state(self):
        check(load().vx_pool_checkpoint(self.h, 1))

    @property
    def stream_ptr(self):
        return int(load().vx_pool_stream(self.h) or 0)


class Server:
    """The served form (vx_server): native threads keep scenes resident in
    pools, admit submissions at round boundaries and step all resident scenes
    of a pool together. With lanes > 1 the scenes are routed by size to one
    pool per lane (REV bounds lane_max_revs, 0 = the defaults)."""

    def __init__(self, ctx: Context, step: VxStepParams, max_slots: int = 64, max_revs: int = 0,
                 hbm_fraction: float = 0.8, lanes: int = 1, lane_max_revs=(0, 0, 0)):
        self.ctx = ctx
        self.h = C.c_void_p()
        cfg = VxServerConfig(max_revs, hbm_fraction, max_slots, step, lanes, (C.c_uint32 * 3)(*lane_max_revs))
        check(load().vx_server_create(ctx.h, C.byref(cfg), C.byref(self.h)))
        self.n = {}

    def submit(self, scene, steps: int, target_velocity=(0.0, 0.0, 0.0), moving=None) -> int:
        """Queues a scene for `steps` fixed steps. `moving` (bool per REV) marks
        targeted REVs whose targets advance at target_velocity (m/s)."""
        keep = {}
        desc = scene_desc(scene, keep)
        mask = np.ascontiguousarray(scene.target_mask, np.uint8).copy()
        if moving is not None:
            mask[np.asarray(moving, bool)] |= 8
        tgt = np.ascontiguousarray(scene.target, np.float64).reshape(-1)
        plan = VxRequestPlan(steps, (C.c_double * 3)(*target_velocity))
        ticket = C.c_uint64()
        check(load().vx_server_submit(self.h, C.byref(desc), _p(mask, C.c_uint8), _p(tgt, C.c_double),
                                      C.byref(plan), C.byref(ticket)))
        self.n[ticket.value] = scene.n
        return ticket.value

    def wait(self, ticket: int, timeout: float = 600.0):
        """(result dict, final positions) once the request has finished, else None."""
        res = VxRequestResult()
        pos = np.zeros(3 * self.n[ticket], np.float64)
        st = load().vx_server_wait(self.h, ticket, timeout, C.byref(res), _p(pos, C.c_double))
        if st == VX_TIMEOUT:
            return None
        check(st)
        self.n.pop(ticket, None)
        return res.as_dict(), pos.reshape(-1, 3)

    def stats(self) -> dict:
        out = VxServerStats()
        check(load().vx_server_get_stats(self.h, C.byref(out)))
        return out.as_dict()

    def close(self):
        if self.h:
            load().vx_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
