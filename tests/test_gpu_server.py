"""The served form (vx_server): continuous batching of resident scenes.

Each request's result must be the same alone and in a mix (bit for bit: pool
slots keep per-scene scalars), requests that arrive while others are stepping
must be admitted and step alongside them, admission must wait for memory, and
moving targets must advance by target_velocity * fixed_dt per step.
"""
import time

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


def step():
    return N.step_params(1e-3, substeps=1, corotation_iterations=2, corotation_tolerance=1e-6, tolerance=1e-8,
                         max_iterations=20000, precision=N.PRECISION_MIXED)


def scenes():
    rng = np.random.default_rng(5)
    return [S.box_union_scene(rng, 8, 24) for _ in range(4)]


def test_result_is_the_same_alone_and_in_a_mix(ctx):
    sc = scenes()
    a = sc[0]
    srv = N.Server(ctx, step(), max_slots=8, max_revs=sum(s.n for s in sc) + 4096)
    alone = srv.wait(srv.submit(a, steps=4))
    assert alone is not None and alone[0]["status"] == N.VX_OK and alone[0]["steps_done"] == 4
    # the same scene again, arriving while three others are already stepping
    others = [srv.submit(s, steps=6) for s in sc[1:]]
    time.sleep(0.05)
    mixed = srv.wait(srv.submit(a, steps=4))
    for t in others:
        r = srv.wait(t)
        assert r is not None and r[0]["status"] == N.VX_OK and r[0]["worst_residual"] <= 1e-8
    assert mixed[0]["status"] == N.VX_OK
    assert np.array_equal(alone[1], mixed[1])
    srv.close()


def test_late_arrivals_step_alongside_running_scenes(ctx):
    sc = scenes()
    srv = N.Server(ctx, step(), max_slots=8, max_revs=sum(s.n for s in sc) + 4096)
    long = srv.submit(sc[1], steps=400)
    deadline = time.time() + 60
    while srv.stats()["scene_steps"] < 5 and time.time() < deadline:  # the long one is running
        time.sleep(0.001)
    short = srv.submit(sc[2], steps=3)
    rs = srv.wait(short)
    assert srv.stats()["resident"] == 1  # the long one is still stepping
    rl = srv.wait(long)
    assert rs[0]["status"] == N.VX_OK and rl[0]["status"] == N.VX_OK
    st = srv.stats()
    # overlapped: fewer rounds than the two requests' steps run one after the other
    assert st["rounds"] < 400 + 3 and st["scene_steps"] == 403
    assert st["completed"] == 2 and st["p99_step_ms"] >= st["p50_step_ms"] > 0.0
    srv.close()


def test_admission_waits_for_memory(ctx):
    sc = scenes()
    big = max(sc, key=lambda s: s.n)
    cap = (big.n + 255) // 256 * 256
    srv = N.Server(ctx, step(), max_slots=8, max_revs=cap)  # room for one copy at a time
    t1 = srv.submit(big, steps=3)
    t2 = srv.submit(big, steps=3)
    r1, r2 = srv.wait(t1), srv.wait(t2)
    assert r1[0]["status"] == N.VX_OK and r2[0]["status"] == N.VX_OK
    # the second copy was admitted only when the first had left
    assert r2[0]["queued_s"] >= 0.9 * r1[0]["run_s"]
    assert np.array_equal(r1[1], r2[1])
    too_big = S.mixed_block(int(np.ceil(cap ** (1 / 3))) + 1, seed=1)
    assert too_big.n > cap
    with pytest.raises(N.VxError):
        srv.submit(too_big, steps=1)  # larger than the whole pool
    srv.close()


def test_moving_targets_advance_with_the_tool(ctx):
    s = S.wood_cube(6)
    top = s.target_mask == 7
    v = (0.0, 0.0, -2e-2)  # m/s: 20 um per 1 ms step
    srv = N.Server(ctx, step(), max_slots=2, max_revs=4096)
    res, x = srv.wait(srv.submit(s, steps=5, target_velocity=v, moving=top))
    assert res["status"] == N.VX_OK
    expect = s.target[top] + 5 * 1e-3 * np.array(v)
    assert np.allclose(x[top], expect, rtol=0, atol=1e-15)
    bottom = s.kinematic == 1
    assert np.array_equal(x[bottom], s.position[bottom])
    srv.close()


def test_blade_cuts_through_contact(ctx):
    """The served scene with a kinematic iron blade driven at 1 m/s into the
    wood: the server steps it with contact and fracture; the blade moved by
    the tool's advance, the wood under its edge was pushed down with it and
    no wood REV is left inside the blade's cross-section below its edge.
    The same request alone and in a mix ends with the same bits."""
    from vxsim import served as V
    rng = np.random.default_rng(21)
    scene, blade = V.served_scene(rng, dof_lo=3e3, dof_hi=6e3)
    other, other_blade = V.served_scene(rng, dof_lo=3e3, dof_hi=6e3)
    p = N.step_params(1e-3, substeps=1, corotation_iterations=2, corotation_tolerance=1e-5, gravity=(0, 0, -9.81),
                      tolerance=1e-8, max_iterations=20000, precision=N.PRECISION_MIXED, fracture=True,
                      contact=True)
    steps = 20
    srv = N.Server(ctx, p, max_slots=4, max_revs=scene.n + other.n + 4096)
    alone = srv.wait(srv.submit(scene, steps, target_velocity=(0.0, 0.0, -1.0), moving=blade))
    t1 = srv.submit(other, steps, target_velocity=(0.0, 0.0, -1.0), moving=other_blade)
    t2 = srv.submit(scene, steps, target_velocity=(0.0, 0.0, -1.0), moving=blade)
    mixed = srv.wait(t2)
    assert srv.wait(t1)[0]["status"] in (N.VX_OK, N.VX_NOT_CONVERGED)
    srv.close()
    res, x = alone
    assert res["status"] in (N.VX_OK, N.VX_NOT_CONVERGED) and res["steps_done"] == steps
    assert np.array_equal(x, mixed[1])
    x0 = scene.position
    # the blade followed its targets: 20 steps of 1 mm
    assert np.allclose(x[blade, 2] - x0[blade, 2], -0.02, atol=1e-9)
    # wood REVs under the edge went down with it
    edge_z = x[blade, 2].min()
    lo = x[blade, :2].min(axis=0) - 0.004
    hi = x[blade, :2].max(axis=0) + 0.004
    wood = ~blade
    under = wood & np.all((x0[:, :2] >= lo) & (x0[:, :2] <= hi), axis=1) & (x0[:, 2] > x0[wood, 2].max() - 0.025)
    assert np.any(under) and np.min(x[under, 2] - x0[under, 2]) < -0.005
    inside = wood & np.all((x[:, :2] > lo + 0.004) & (x[:, :2] < hi - 0.004), axis=1) & (x[:, 2] > edge_z + 0.005)
    assert not np.any(inside)


def test_lanes_route_by_size_and_keep_results(ctx):
    """Two lanes (scenes up to 2,000 REVs, and larger): every request ends with
    the same bits as on a one-lane server, and the small scenes finish while
    the large ones still run their own rounds."""
    sc = scenes()
    sizes = [s.n for s in sc]
    assert min(sizes) <= 2000 < max(sizes), sizes
    cap = sum(sizes) + 8192

    def run(lanes):
        srv = N.Server(ctx, step(), max_slots=8, max_revs=4 * cap, lanes=lanes, lane_max_revs=(2000, 0, 0))
        tickets = [srv.submit(s, steps=3) for s in sc]
        out = [srv.wait(t) for t in tickets]
        st = srv.stats()
        srv.close()
        return out, st

    one, _ = run(1)
    two, st = run(2)
    assert st["completed"] == len(sc) and st["failed"] == 0
    for (r1, x1), (r2, x2) in zip(one, two):
        assert r1["status"] == r2["status"] == N.VX_OK and r2["steps_done"] == 3
        assert np.array_equal(x1, x2)
