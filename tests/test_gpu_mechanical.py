"""The device step (vx_scene_step with the fracture stage) through the
reference's 10^3 tension fixture (src/experiments.rs:51-108), against the
oracle's step and the recorded regression (validation/mechanical-tests.txt:3).

The device runs the FP64 solve with the CPU path's rules (PCG cap 300, 1e-5,
block-Jacobi factor of the first pass reused), so it takes the oracle's
iteration counts; the reaction is read from the bond workspace last_force the
fracture commit evaluates (vx_scene_get_last_forces).
"""
import pytest

from vxsim import native as N
import mechanical_fixture as MF
from test_oracle_mechanical import OracleRamp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def device_ramp(ctx):
    params = N.step_params(MF.DT, corotation_iterations=MF.COROTATION_ITERATIONS,
                           corotation_tolerance=MF.COROTATION_TOLERANCE, tolerance=MF.TOLERANCE,
                           max_iterations=MF.PCG_CAP, precision=N.PRECISION_FP64, reuse=True, fracture=True)

    class DeviceRamp:
        def __init__(self, scene):
            self.d = N.DeviceScene(ctx, scene)

        def set_targets(self, mask, target):
            self.d.set_targets(mask, target)

        def step(self):
            st = self.d.step(params)
            assert st["status"] in (N.VX_OK, N.VX_NOT_CONVERGED), st
            return st["broken"]

        def last_forces(self):
            return self.d.last_forces()

    return DeviceRamp


def test_tension_on_the_device_matches_oracle_and_record(ctx):
    g = MF.run_test(device_ramp(ctx), "tension")
    o = MF.run_test(OracleRamp, "tension")
    rec = MF.RECORDED["tension"]
    print(f"tension on the device: parallel {g['parallel']:.3f} N, perpendicular {g['perpendicular']:.3f} N, "
          f"ratio {g['ratio']:.3f}, first breaks {g['breaks']} at steps {g['steps']}; oracle "
          f"{o['parallel']:.3f} / {o['perpendicular']:.3f} N; recorded {rec['parallel']:.3f} / "
          f"{rec['perpendicular']:.3f} N")
    assert g["breaks"] == o["breaks"] == rec["breaks"]
    assert g["steps"] == o["steps"]
    # last_force is stored in f32 as the reference's workspace is
    for k in ("parallel", "perpendicular"):
        assert abs(g[k] - o[k]) <= 1e-6 * o[k]
        assert abs(g[k] - rec[k]) <= 1e-4 * rec[k]
