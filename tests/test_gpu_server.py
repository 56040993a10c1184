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
