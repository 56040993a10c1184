"""The fixed step on the device (vx_scene_step) against the oracle's restatement
of solver::step_with_axis_targets_and_loads (vxo_step), without fracture."""
import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N, scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("substeps,passes", [(1, 1), (2, 3)])
def test_step_matches_oracle_under_gravity(ctx, substeps, passes):
    s = S.mixed_block(8, seed=2)
    g = (0.0, 0.0, -9.81)
    # corotation_tolerance 0: every pass runs on both sides (an early exit on
    # an angle change near the bound could differ by one pass)
    o = O.OracleStepper(s, fixed_dt=1e-3, substeps=substeps, iterations=20000, solver_tolerance=1e-14,
                        corotation_tolerance=0.0, corotation_iterations=passes, gravity=g, fracture=False)
    d = N.DeviceScene(ctx, s)
    p = N.step_params(1e-3, substeps=substeps, corotation_iterations=passes, corotation_tolerance=0.0, gravity=g,
                      tolerance=1e-14, max_iterations=20000, precision=N.PRECISION_FP64, reuse=True)
    for _ in range(3):
        o.step()
        st = d.step(p)
        assert st["status"] == N.VX_OK and st["converged"] == 1, st
    # Both sides are FP64 with the same PCG iteration counts, but round
    # differently (fused multiply-adds and reduction order on the GPU, none
    # in the oracle); the stiffness contrast of the block amplifies that to
    # ~1e-9 of the displacement. The supported block settles, so its
    # velocities shrink towards zero: they are compared against the run's
    # characteristic velocity (displacement / elapsed time).
    disp = o.positions - s.position
    assert rel(d.positions() - s.position, disp) < 1e-8
    v_scale = np.linalg.norm(disp) / 3e-3
    assert np.linalg.norm(d.velocities() - o.velocity.reshape(-1, 3)) < 1e-7 * v_scale
    d.close()


def test_step_drives_targets_and_stops_early(ctx):
    """The wood cube's top layer is targeted: after a step the targeted axes sit
    on their targets with velocity (x - previous) / h, and the passes stop once
    the fit no longer moves (fewer passes than allowed)."""
    s = S.wood_cube(6)
    o = O.OracleStepper(s, fixed_dt=1e-3, substeps=1, iterations=20000, solver_tolerance=1e-10,
                        corotation_tolerance=1e-3, corotation_iterations=4, fracture=False)
    d = N.DeviceScene(ctx, s)
    p = N.step_params(1e-3, corotation_iterations=4, corotation_tolerance=1e-3, tolerance=1e-10,
                      max_iterations=20000, precision=N.PRECISION_FP64, reuse=True)
    o.step()
    st = d.step(p)
    assert st["passes"] < 4
    top = np.nonzero(s.target_mask == 7)[0]
    x = d.positions()
    assert np.allclose(x[top], s.target[top], rtol=0, atol=1e-15)
    v = d.velocities()
    assert np.allclose(v[top], (s.target[top] - s.position[top]) / 1e-3, rtol=1e-12, atol=1e-15)
    assert rel(x - s.position, o.positions - s.position) < 1e-8
    d.close()


def test_mixed_precision_step_meets_the_fp64_target(ctx):
    s = S.mixed_block(12, seed=4)
    d = N.DeviceScene(ctx, s)
    p = N.step_params(1e-3, corotation_iterations=2, gravity=(0.0, 0.0, -9.81), tolerance=1e-8,
                      max_iterations=20000, precision=N.PRECISION_MIXED)
    st = d.step(p)
    assert st["status"] == N.VX_OK and st["residual"] <= 1e-8
    d.close()


def test_velocity_set_and_impulse_keep_targeted_axes_at_zero(ctx):
    s = S.wood_cube(4)
    d = N.DeviceScene(ctx, s)
    free = int(np.nonzero((s.kinematic == 0) & (s.target_mask == 0))[0][0])
    tgt = int(np.nonzero(s.target_mask == 7)[0][0])
    d.update_velocities([free, tgt], [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
    d.update_velocities([free], [[0.5, 0.5, 0.5]], add=True)
    v = d.velocities()
    assert np.array_equal(v[free], [1.5, 2.5, 3.5])
    assert np.array_equal(v[tgt], [0.0, 0.0, 0.0])
    with pytest.raises(N.VxError):
        d.update_velocities([s.n], [[0.0, 0.0, 0.0]])
    d.close()


@pytest.mark.parametrize("edge", [1, 3])
def test_odd_rev_counts(ctx, edge):
    """Scenes with an odd REV count (1 and 27): the FP32 stiffness arrays keep
    every axis on a 16-byte boundary, and passes and steps match the oracle."""
    s = S.wood_cube(edge) if edge > 1 else S.from_cells(np.zeros((1, 3), np.int32), 1, S.M.table(),
                                                          anisotropy=1.0)
    assert s.n % 2 == 1
    if edge == 1:
        h, m = 0.01, float(s.mass[0])
        s.loads[:] = [[3.0 * m, 2.0 * m, 0.0]]
        d = N.DeviceScene(ctx, s)
        p = N.step_params(h, substeps=1, corotation_iterations=1, tolerance=1e-5, max_iterations=1)
        st = d.step(p)
        assert st["status"] == N.VX_OK
        assert np.allclose(d.velocities()[0], [0.03, 0.02, 0.0], rtol=0, atol=1e-12)
        d.close()
        return
    top = s.target_mask == 7
    s.position[top] = s.target[top]  # targeted REVs on their targets, as after a prediction
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3, predicted=s.position)
    o.factor_block_jacobi()
    ref, _, _ = o.pcg(20000, 1e-14)
    for precision, kernel in ((N.PRECISION_FP64, N.KERNEL_AUTO), (N.PRECISION_MIXED, N.KERNEL_STREAMING),
                              (N.PRECISION_MIXED, N.KERNEL_PERSISTENT)):
        d = N.DeviceScene(ctx, s)
        d.fit_rotations()
        d.set_predicted(s.position)
        st = d.corotational_pass(1e-3, 1e-12 if precision == N.PRECISION_FP64 else 1e-8, 20000,
                                 precision=precision, kernel=kernel)
        assert st["converged"] == 1, (precision, kernel, st)
        assert rel(d.positions() - s.position, ref.reshape(-1, 3)) < (1e-9 if precision == N.PRECISION_FP64 else 1e-6)
        d.close()
