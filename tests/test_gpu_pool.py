"""The scene pool (batched and served forms) against single-scene solves.

A pooled scene's pass must give the single scene's answer within the stated
1e-8 target, be bit-identical whether it is alone in the pool or solved with
other scenes, leave slots outside the call untouched, and refuse scenes that
do not fit (admission by footprint).
"""
import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu

H, TOL, CAP = 1e-3, 1e-8, 50000


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def scenes():
    rng = np.random.default_rng(11)
    return [S.mixed_block(8, seed=1), S.wood_cube(), S.box_union_scene(rng, 8, 20), S.mixed_block(12, seed=3)]


def single(ctx, scene):
    d = N.DeviceScene(ctx, scene)
    d.fit_rotations()
    st = d.corotational_pass(H, TOL, CAP, precision=N.PRECISION_MIXED)
    x = d.positions()
    d.close()
    return x, st


def test_pool_pass_matches_single_scene_solves(ctx):
    sc = scenes()
    pool = N.DevicePool(ctx, sum(s.n for s in sc) + 4096, 8)
    slots = [pool.add(s) for s in sc]
    pool.fit_rotations()
    status, stats = pool.corotational_pass(H, TOL, CAP)
    assert status == N.VX_OK
    for s, k in zip(sc, slots):
        assert stats[k]["converged"] == 1 and stats[k]["true_residual"] <= TOL, stats[k]
        x1, st1 = single(ctx, s)
        x0 = s.position
        # both meet 1e-8 against the FP64 operator; they agree to the solve error
        assert rel(pool.positions(k) - x0, x1 - x0) < 1e-5
    pool.close()


def test_pool_scene_is_bit_identical_alone_and_in_a_mix(ctx):
    sc = scenes()
    alone = N.DevicePool(ctx, 1 << 16, 4)
    a = alone.add(sc[0])
    alone.fit_rotations()
    alone.corotational_pass(H, TOL, CAP)
    mix = N.DevicePool(ctx, 1 << 17, 8)
    others = [mix.add(s) for s in sc[1:3]]
    b = mix.add(sc[0])
    mix.add(sc[3])
    mix.fit_rotations()
    mix.corotational_pass(H, TOL, CAP)
    assert np.array_equal(alone.positions(a), mix.positions(b))
    assert np.array_equal(alone.rotations(a), mix.rotations(b))
    alone.close()
    mix.close()


def test_disabled_slots_are_untouched_and_rotations_match(ctx):
    sc = scenes()
    pool = N.DevicePool(ctx, 1 << 17, 8)
    slots = [pool.add(s) for s in sc]
    before = pool.positions(slots[1]).copy()
    angles = pool.fit_rotations(enabled=[slots[0], slots[2]])
    assert angles[slots[1]] == 0.0
    pool.corotational_pass(H, TOL, CAP, enabled=[slots[0], slots[2]])
    assert np.array_equal(pool.positions(slots[1]), before)
    d = N.DeviceScene(ctx, sc[0])
    ang = d.fit_rotations()
    assert abs(ang - angles[slots[0]]) <= 1e-12 * max(ang, 1e-30)
    d.close()
    pool.close()


def test_pool_admission_and_slot_reuse(ctx):
    big = S.mixed_block(16, seed=2)     # 4096 REVs = 16 tiles
    small = S.wood_cube()               # 1000 REVs = 4 tiles
    pool = N.DevicePool(ctx, 20 * 256, 4)
    a = pool.add(big)
    b = pool.add(small)
    with pytest.raises(N.VxError) as e:
        pool.add(S.mixed_block(8, seed=9))  # 512 REVs: no 2-tile range left
    assert e.value.status == N.VX_OOM
    pool.remove(b)
    c = pool.add(S.mixed_block(8, seed=9))
    assert c == b
    pool.fit_rotations()
    status, stats = pool.corotational_pass(H, TOL, CAP)
    assert status == N.VX_OK and stats[c]["converged"] == 1
    x1, _ = single(ctx, S.mixed_block(8, seed=9))
    x0 = S.mixed_block(8, seed=9).position
    assert rel(pool.positions(c) - x0, x1 - x0) < 1e-5
    pool.close()


def test_pool_bond_stress_matches_single_scene(ctx):
    s = S.mixed_block(8, seed=4)
    pool = N.DevicePool(ctx, 1 << 14, 2)
    k = pool.add(S.wood_cube())
    j = pool.add(s)
    pool.fit_rotations()
    pool.corotational_pass(H, 1e-12, CAP)
    d = N.DeviceScene(ctx, s)
    d.set_positions(pool.positions(j))
    d.set_rotations(pool.rotations(j))
    d.corotational_pass(H, 1e-12, 10)  # assembles the same frames; positions then reset
    d.set_positions(pool.positions(j))
    g = d.bond_stress()
    p = pool.bond_stress(j)
    assert np.array_equal(g["ratio"] < 0, p["ratio"] < 0)
    live = g["ratio"] >= 0
    assert np.all(np.abs(g["ratio"][live] - p["ratio"][live]) <= 1e-5 * np.maximum(g["ratio"][live], 1e-3))
    d.close()
    pool.close()


def step_params(kernel=N.KERNEL_AUTO):
    return N.step_params(1e-3, substeps=2, corotation_iterations=3, corotation_tolerance=1e-6,
                         gravity=(0.0, 0.0, -9.81), tolerance=TOL, max_iterations=CAP,
                         precision=N.PRECISION_MIXED, kernel=kernel)


def test_pool_step_matches_single_scene_steps(ctx):
    """vx_pool_step against vx_scene_step on each scene over three steps. Both
    reach 1e-8 in every pass, so they agree to the solve error: the pool runs
    the classic recurrence, the single scene the on-chip Chronopoulos-Gear one,
    so the two stop at different points inside the 1e-8 ball, and six passes
    give a relative difference up to about kappa * 1e-8 (measured 1.6e-5 on the
    8^3 block); the bar is 5e-5."""
    sc = scenes()
    pool = N.DevicePool(ctx, sum(s.n for s in sc) + 4096, 8)
    slots = [pool.add(s) for s in sc]
    p = step_params()
    for _ in range(3):
        status, stats = pool.step(p)
        assert status == N.VX_OK
        for k in slots:
            assert stats[k]["converged"] == 1 and stats[k]["residual"] <= TOL, stats[k]
    for s, k in zip(sc, slots):
        d = N.DeviceScene(ctx, s)
        for _ in range(3):
            assert d.step(p)["status"] == N.VX_OK
        x0 = s.position
        assert rel(pool.positions(k) - x0, d.positions() - x0) < 5e-5
        # velocities are (x - predicted) / h: a position difference within the
        # bar above, divided by the substep h = 0.5 ms
        v_bar = 5e-5 * np.linalg.norm(d.positions() - x0) / 5e-4
        assert np.linalg.norm(pool.velocities(k) - d.velocities()) <= v_bar
        d.close()
    pool.close()


@pytest.mark.parametrize("kernel", [N.KERNEL_AUTO, N.KERNEL_PERSISTENT])
def test_pool_step_is_bit_identical_alone_and_in_a_mix(ctx, kernel):
    """A scene stepped alone in a pool and the same scene stepped together
    with others (admitted at a different slot and tile range) end with the
    same bits after three steps, velocities included: with the tile kernels,
    and with persistent waves, where the others also change the wave's
    largest block (one kernel instantiation serves every wave for this)."""
    sc = scenes()
    target = sc[2]
    p = step_params(kernel)
    alone = N.DevicePool(ctx, target.n + 4096, 4)
    ka = alone.add(target)
    mixed = N.DevicePool(ctx, sum(s.n for s in sc) + 4096, 8)
    others = [mixed.add(s) for s in sc[:2]]
    km = mixed.add(target)
    mixed.add(sc[3])
    for _ in range(3):
        assert alone.step(p)[0] == N.VX_OK
        assert mixed.step(p)[0] == N.VX_OK
    assert np.array_equal(alone.positions(ka), mixed.positions(km))
    assert np.array_equal(alone.velocities(ka), mixed.velocities(km))
    assert others
    alone.close()
    mixed.close()


def test_sharded_front_end_gives_each_scene_its_pool_result(ctx):
    """vxsim.sharding with this process as the only rank: the batch goes to one
    pool through sharding.pool_pass, and every scene's displacement is the bits
    of the same scene solved alone in a pool (slots do not interact)."""
    from vxsim import sharding as Hs
    sc = scenes()
    out = Hs.solve_sharded(sc, Hs.pool_pass(ctx, h=H, tolerance=TOL, max_iterations=CAP))
    assert len(out) == len(sc)
    for s, res in zip(sc, out):
        assert res["stats"]["converged"] == 1 and res["stats"]["true_residual"] <= TOL
        alone = N.DevicePool(ctx, 1 << 16, 2)
        k = alone.add(s)
        alone.fit_rotations()
        alone.corotational_pass(H, TOL, CAP)
        assert np.array_equal(alone.positions(k) - s.position, res["displacement"])
        alone.close()


def test_persistent_waves_match_the_tile_kernels(ctx):
    """The pool's inner solves in waves of the persistent kernel (one cooperative
    launch per wave, per-slot reductions and convergence masks) against the
    chunk graph of tile kernels: both reach 1e-8 per slot and take the same
    inner iterations, and the displacements agree to the solve error."""
    sc = scenes()
    out = {}
    for kernel in (N.KERNEL_STREAMING, N.KERNEL_PERSISTENT):
        pool = N.DevicePool(ctx, sum(s.n for s in sc) + 4096, 8)
        slots = [pool.add(s) for s in sc]
        pool.fit_rotations()
        status, stats = pool.corotational_pass(H, TOL, CAP, kernel=kernel)
        assert status == N.VX_OK
        out[kernel] = [(pool.positions(k) - s.position, stats[k]) for s, k in zip(sc, slots)]
        pool.close()
    for (d_s, st_s), (d_p, st_p) in zip(out[N.KERNEL_STREAMING], out[N.KERNEL_PERSISTENT]):
        assert st_s["converged"] == 1 and st_p["converged"] == 1
        assert st_p["true_residual"] <= TOL and st_s["true_residual"] <= TOL
        assert abs(st_p["iterations"] - st_s["iterations"]) <= 0.02 * st_s["iterations"] + 4
        assert rel(d_p, d_s) < 2e-5


def test_persistent_waves_of_many_slots(ctx):
    """More slots than fit one wave (each 16^3 slot takes 3 blocks of at most
    1,536 REVs, so 60 slots need two waves of at most 148 blocks): every slot
    converges and equals the same scene solved alone in a pool, bit for bit."""
    s = S.mixed_block(16, seed=9)
    pool = N.DevicePool(ctx, 60 * s.n + 4096, 64)
    slots = [pool.add(s) for _ in range(60)]
    pool.fit_rotations()
    status, stats = pool.corotational_pass(H, TOL, CAP, kernel=N.KERNEL_PERSISTENT)
    assert status == N.VX_OK and all(stats[k]["converged"] == 1 for k in slots)
    alone = N.DevicePool(ctx, s.n + 4096, 2)
    a = alone.add(s)
    alone.fit_rotations()
    alone.corotational_pass(H, TOL, CAP, kernel=N.KERNEL_PERSISTENT)
    ref = alone.positions(a)
    assert all(np.array_equal(pool.positions(k), ref) for k in slots)
    alone.close()
    pool.close()
