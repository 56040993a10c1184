"""The fracture stage on the device (vx_fracture_commit, inside vx_scene_step)
against the oracle's fracture::update restatement run by vxo_step.

A 6^3 wood cube (grain +Z) is pulled 10 mm at its top layer: the 144
grain-aligned bonds yield and gain damage every 1 ms step (0.16, 0.35, 0.54,
0.73, 0.92 in the oracle) and all break in the sixth. The
device keeps the bond state in f32 as the reference does (the oracle in f64),
so damage and plastic strain agree to f32 rounding; the broken-bond sets must
be identical except for bonds within 1e-6 of their limit.
"""
import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_fracture_steps_match_the_oracle(ctx):
    s = S.wood_cube(6, displacement=1e-2)
    steps = 6
    o = O.OracleStepper(s, fixed_dt=1e-3, substeps=1, iterations=20000, solver_tolerance=1e-13,
                        corotation_tolerance=0.0, corotation_iterations=2, fracture=True)
    d = N.DeviceScene(ctx, s)
    p = N.step_params(1e-3, corotation_iterations=2, corotation_tolerance=0.0, tolerance=1e-13,
                      max_iterations=20000, precision=N.PRECISION_FP64, reuse=True, fracture=True)
    broken = 0
    heat = 0.0
    for _ in range(steps):
        o.step()
        st = d.step(p)
        assert st["status"] == N.VX_OK, st
        broken += st["broken"]
        heat += sum(st["dissipation"].values())
    n = s.n
    ob = o.bonds
    dmg_o = np.array([ob[e].damage for e in range(3 * n)]).reshape(3, n)
    pl_o = np.array([list(ob[e].plastic) for e in range(3 * n)]).reshape(3, n, 3)
    nb_o = np.array([ob[e].neighbor for e in range(3 * n)], np.uint32).reshape(3, n)
    bs = d.bond_state()
    assert o.broken > 0 and broken == o.broken
    assert np.array_equal(d.neighbors(), nb_o)
    assert np.max(np.abs(bs["damage"] - dmg_o)) <= 1e-5
    assert np.max(np.abs(bs["plastic"] - pl_o)) <= 1e-6 * max(np.max(np.abs(pl_o)), 1e-12) + 1e-9
    assert rel(d.positions() - s.position, o.positions - s.position) < 1e-5
    total_o = o.d.plastic_heat + o.d.stored_plastic + o.d.surface_work + o.d.damage_heat + o.d.pending_release
    assert heat > 0 and abs(heat - total_o) <= 1e-4 * total_o
    d.close()


def test_commit_is_deterministic_and_needs_an_assembly(ctx):
    s = S.wood_cube(4, displacement=1e-3)
    d = N.DeviceScene(ctx, s)
    with pytest.raises(N.VxError):
        d.fracture_commit(1e-3)
    d.fit_rotations()
    d.corotational_pass(1e-3, 1e-10, 20000, precision=N.PRECISION_FP64)
    d.save_state()
    first = d.fracture_commit(1e-3)
    d.close()
    d2 = N.DeviceScene(ctx, s)
    d2.fit_rotations()
    d2.corotational_pass(1e-3, 1e-10, 20000, precision=N.PRECISION_FP64)
    second = d2.fracture_commit(1e-3)
    assert first == second  # the same bits
    d2.close()
