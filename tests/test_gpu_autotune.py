"""The autotuner (vx_scene_autotune): it times every candidate launch
configuration of the inner solve, keeps the fastest for later passes (which
still reach their target), and stores / reuses its choice in a cache file."""
import numpy as np
import pytest

from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("precision,edge", [(N.PRECISION_MIXED, 24), (N.PRECISION_MIXED, 80),
                                            (N.PRECISION_FP64, 40)])
def test_tuner_keeps_the_fastest_candidate(ctx, tmp_path, precision, edge):
    s = S.damaged_lattice(edge, seed=4)
    d = N.DeviceScene(ctx, s)
    d.set_predicted(s.position)
    d.fit_rotations()
    tol = 1e-8 if precision == N.PRECISION_MIXED else 1e-10
    assert d.corotational_pass(1e-3, tol, 50000, precision=precision)["converged"] == 1
    cache = tmp_path / "tune.txt"
    res = d.autotune(precision, cache)
    cands = res["candidates"]
    assert res["from_cache"] == 0 and len(cands) >= 3
    assert all(np.isfinite(us) and us > 0 for _, _, us in cands)
    best = min(cands, key=lambda c: c[2])
    assert (res["kernel"], res["blocks_per_sm"]) == (best[0], best[1])
    if precision == N.PRECISION_MIXED and edge <= 60:
        # the persistent forms: the brick plan with 1 or 2 threads per REV and
        # tiles of >= 256 or >= 128 REVs, the range plan with two grid
        # reductions per iteration at 512, 608, 768 or 896 threads per block,
        # and with one
        forms = {b for k, b, _ in cands if k == N.KERNEL_PERSISTENT}
        assert forms == {1, 2, 3, 4, 5, 6, 7, 8, 9}, cands
    print({N.tune_label(k, b): round(us, 2) for k, b, us in cands})
    # later passes run with the choice and still reach the target
    d.fit_rotations()
    st = d.corotational_pass(1e-3, tol, 50000, precision=precision, reuse=True)
    assert st["converged"] == 1 and st["true_residual"] <= tol * 10
    d.close()
    # a second scene of the same size reuses the stored choice without timing
    d2 = N.DeviceScene(ctx, s)
    d2.set_predicted(s.position)
    d2.fit_rotations()
    d2.corotational_pass(1e-3, tol, 50000, precision=precision)
    again = d2.autotune(precision, cache)
    assert again["from_cache"] == 1 and (again["kernel"], again["blocks_per_sm"]) == (best[0], best[1])
    assert cache.read_text().count("\n") == 1
    d2.close()


def test_tuner_needs_an_assembled_scene(ctx):
    d = N.DeviceScene(ctx, S.wood_cube(4))
    with pytest.raises(N.VxError):
        d.autotune(N.PRECISION_MIXED)
    d.close()
