"""The oracle's step against the reference's recorded mechanical regression
(validation/mechanical-tests.txt:3-4), the 10^3 axial fixture of
src/experiments.rs:51-108 restated in mechanical_fixture.py.

Tension is reproduced: the recorded run is the reference's f32 CPU solver with
its default IC(0) preconditioner, the oracle is FP64 with block-Jacobi, both
stop each PCG at a relative residual of 1e-5. The peaks then agree to about
1e-5 relative: the first break comes at the same ramp step (217 parallel, 18
perpendicular), and the f32 positions near z = 1 m (spacing 1.2e-7 m against
1e-4 m of bond elongation) and the two preconditioners' different 1e-5
solves bound the agreement at a few 1e-5; the bar is 1e-4.

Compression is not reproduced: the restatement fails uniformly at the
compression limits (all 900 grain-wise bonds in one step, 521,709 N parallel
and 20,160 N perpendicular), where the recorded run broke 3 and 4 bonds at
284,145 N and 8,732 N. The oracle's result does not move with the PCG
tolerance (1e-3 to 1e-10), with the contact stage on, or with f32-sized
perturbations of the start positions; the recorded localisation is not
explained by anything on this path. The test states it as an expected failure.
"""
import pytest

import pyoracle as O
import mechanical_fixture as MF


class OracleRamp:
    def __init__(self, scene):
        self.o = O.OracleStepper(scene, fixed_dt=MF.DT, substeps=1, iterations=MF.PCG_CAP,
                                 solver_tolerance=MF.TOLERANCE, corotation_tolerance=MF.COROTATION_TOLERANCE,
                                 corotation_iterations=MF.COROTATION_ITERATIONS, fracture=True)
        self.seen = 0

    def set_targets(self, mask, target):
        self.o.set_targets(mask, target)

    def step(self):
        self.o.step()
        broken = self.o.broken - self.seen
        self.seen = self.o.broken
        return broken

    def last_forces(self):
        return self.o.last_forces()


def test_tension_matches_the_recorded_regression():
    r = MF.run_test(OracleRamp, "tension")
    rec = MF.RECORDED["tension"]
    print(f"tension: parallel {r['parallel']:.3f} N (recorded {rec['parallel']:.3f}), perpendicular "
          f"{r['perpendicular']:.3f} N (recorded {rec['perpendicular']:.3f}), ratio {r['ratio']:.3f} "
          f"(recorded {rec['ratio']:.3f}), first breaks {r['breaks']} at steps {r['steps']}")
    assert r["breaks"] == rec["breaks"]
    assert abs(r["parallel"] - rec["parallel"]) <= 1e-4 * rec["parallel"]
    assert abs(r["perpendicular"] - rec["perpendicular"]) <= 1e-4 * rec["perpendicular"]
    assert abs(r["ratio"] - rec["ratio"]) <= 2e-3


def test_compression_fails_at_the_limits_in_the_restatement():
    r = MF.run_test(OracleRamp, "compression")
    # grain-wise bonds fail together once the hardened yield reaches 50 MPa
    # (parallel) and at the 2 MPa perpendicular limit: 100 bonds x 1e-4 m^2
    assert r["breaks"] == (900, 900)
    assert 5.0e5 < r["parallel"] < 5.4e5 and 2.0e4 < r["perpendicular"] < 2.05e4


@pytest.mark.xfail(strict=True, reason="the recorded compression run localised (3/4 first breaks at 0.55x and "
                                       "0.43x of the uniform limits); the restatement fails uniformly")
def test_compression_matches_the_recorded_regression():
    r = MF.run_test(OracleRamp, "compression")
    rec = MF.RECORDED["compression"]
    assert r["breaks"] == rec["breaks"]
    assert abs(r["ratio"] - rec["ratio"]) <= 2e-3
