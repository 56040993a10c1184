"""The reference's 10^3 axial loading fixture (src/experiments.rs:14-108),
restated for the oracle's step and the device's step.

A 10x10x10 specimen of the built-in wood (10/0.6 GPa, 650 kg/m^3), grain along
X ("parallel") or Z ("perpendicular"), is lifted 1 m in Z (f32, as the fixture
does), then pulled (sign +1) or compressed (sign -1) along X: the x = min layer
is held at rest and the x = max layer targeted at rest + 0.12 (max - min) n / 500
in step n = 1..500. Each step is solver::step_with_targets with the scene file's
settings (dt 1 ms, one substep, corotation 4 passes at 1e-5, PCG cap 300 at
1e-5, the wood_chop fracture settings). The reaction is the |x| component of the
summed last forces of the bonds that cross the right grip (`reaction`,
src/experiments.rs:32-49); the run stops at the first step that breaks a bond.

Recorded by the reference (validation/mechanical-tests.txt:3-4, f32 CPU solver):
tension parallel 1,022,767.250 N, perpendicular 25,920.164 N, ratio 39.458,
first breaks 900/900; compression parallel 284,145.156 N, perpendicular
8,732.482 N, ratio 32.539, first breaks 3/4.
"""
from __future__ import annotations

import numpy as np

from vxsim import materials as M
from vxsim import scenes as S

RECORDED = {
    "tension": {"parallel": 1022767.250, "perpendicular": 25920.164, "ratio": 39.458, "breaks": (900, 900)},
    "compression": {"parallel": 284145.156, "perpendicular": 8732.482, "ratio": 32.539, "breaks": (3, 4)},
}
STEPS = 500
DT = 1e-3
PCG_CAP = 300          # SceneConfig::iterations set by the fixture (CPU solve)
TOLERANCE = 1e-5       # solver_relative_tolerance of scenes/wood_chop.ron
COROTATION_ITERATIONS = 4
COROTATION_TOLERANCE = 1e-5


def specimen(fiber) -> S.Scene:
    """`specimen([10, 10, 10], fiber)`: Scene::new of the 10^3 trunk with the
    built-in material table, then every position lifted by +1 m in f32."""
    s = S.scene_new((10, 10, 10), fibers=tuple(float(v) for v in fiber), anisotropy=1.0,
                    materials_table=M.table())
    p32 = np.asarray(s.position, np.float32)
    p32[:, 2] = p32[:, 2] + np.float32(1.0)
    s.position = p32.astype(np.float64)
    return s


def grips(rest32: np.ndarray):
    x = rest32[:, 0]
    lo, hi = x.min(), x.max()
    tenth = np.float32(0.01) * np.float32(0.1)
    return x < lo + tenth, x > hi - tenth, lo, hi


def ramp_targets(rest32, left, right, lo, hi, sign, n):
    """Targets of step n: the left grip at rest, the right grip displaced in x (f32)."""
    disp = np.float32(sign) * (hi - lo) * np.float32(0.12) * np.float32(n) / np.float32(STEPS)
    target = rest32.copy()
    target[right, 0] = rest32[right, 0] + disp
    mask = np.where(left | right, 7, 0).astype(np.uint8)
    return mask, target.astype(np.float64)


def reaction(neighbor_rest: np.ndarray, last_force: np.ndarray, grip: np.ndarray) -> float:
    """|x| of the summed last forces on the grip: + for bonds owned by a grip REV,
    - for bonds whose partner is one (the rest topology, broken bonds included)."""
    n = grip.size
    f = 0.0
    for a in range(3):
        nb = neighbor_rest[a]
        has = nb != S.EMPTY
        owner = np.arange(n)
        fx = last_force[a, :, 0].astype(np.float64)
        f += fx[has & grip[owner]].sum()
        partner_grip = np.zeros(n, bool)
        partner_grip[has] = grip[nb[has]]
        f -= fx[has & partner_grip].sum()
    return abs(f)


def run_axial(stepper, fiber, sign) -> dict:
    """Drive `stepper` (an object with set_targets(mask, target), step() -> broken
    bonds of the step, last_forces() -> (3, n, 3)) through the ramp."""
    s = specimen(fiber)
    rest32 = np.asarray(s.position, np.float32)
    left, right, lo, hi = grips(rest32)
    nbr_rest = s.neighbor.copy()
    st = stepper(s)
    peak = 0.0
    for n in range(1, STEPS + 1):
        mask, target = ramp_targets(rest32, left, right, lo, hi, sign, n)
        st.set_targets(mask, target)
        broken = st.step()
        peak = max(peak, reaction(nbr_rest, st.last_forces(), right))
        if broken > 0:
            return {"peak": peak, "breaks": broken, "step": n}
    return {"peak": peak, "breaks": 0, "step": STEPS}


def run_test(stepper, kind: str) -> dict:
    sign = 1.0 if kind == "tension" else -1.0
    par = run_axial(stepper, (1.0, 0.0, 0.0), sign)
    perp = run_axial(stepper, (0.0, 0.0, 1.0), sign)
    return {"parallel": par["peak"], "perpendicular": perp["peak"], "ratio": par["peak"] / perp["peak"],
            "breaks": (par["breaks"], perp["breaks"]), "steps": (par["step"], perp["step"])}
