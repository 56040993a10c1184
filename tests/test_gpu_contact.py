"""Contact projection and contact velocities on the device (vx_contact.cu)
against the oracle's restatement of collision::project and
resolve_velocities_with_precontact (src/collision.rs).

Both sides compute in FP64 from the same inputs and the device rounds every
expression as written (no fused multiply-adds), so the corrected positions,
the contacts, the pair counts and the velocities must be bit-identical; the
heat totals are sums in a different order and agree to 1e-12. The cases are
the reference's own collision tests, a rubble of unbonded REVs with many
overlapping and crossing pairs, fast REVs whose swept boxes take the
large-box path, deep overlaps whose corrections exceed the replay's movement
bound, and the step with contact against the oracle's step."""
import math

import numpy as np
import pytest

import pyoracle as O
from vxsim import materials as M
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu

CELL = float(np.float32(0.01))


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _device(ctx, s, pos, prev, tmask=None):
    """A device scene created at the scene's rest positions, then moved."""
    d = N.DeviceScene(ctx, s)
    d.write_field(N.FIELD_POSITION, pos)
    d.write_field(N.FIELD_PREVIOUS, prev)
    if tmask is not None:
        d.set_targets(tmask, pos)
    return d


def _check_project(ctx, s, pos, prev, tmask=None):
    op, oq, oc, ost = O.contact_project(pos, prev, s.position, s.kinematic, s.mass.astype(np.float64), s.neighbor,
                                        tmask)
    d = _device(ctx, s, pos, prev, tmask)
    st = d.contact_project()
    dp = d.positions()
    dq = d.read_field(N.FIELD_PREVIOUS)
    dc = d.contacts()
    assert st["candidates"] == ost["candidates"] and st["pairs"] == ost["pairs"], (st, ost)
    assert st["contacts"] == len(oc)
    assert st["sweeps"] == ost["sweeps"], (st, ost)
    assert np.array_equal(dc["i"], oc["i"]) and np.array_equal(dc["j"], oc["j"])
    assert np.array_equal(dc["normal"], oc["normal"]) and np.array_equal(dc["new_impact"], oc["new_impact"])
    assert np.array_equal(dp, op), np.max(np.abs(dp - op))
    assert np.array_equal(dq, oq), np.max(np.abs(dq - oq))
    return d, st, oc


def test_set_previous_writes_every_rev(ctx):
    s = S.from_cells(S.grid_cells(4, 3, 2), M.component_id("iron"), M.table())
    rng = np.random.default_rng(3)
    prev = s.position + rng.normal(0, 1e-3, s.position.shape)
    d = N.DeviceScene(ctx, s)
    d.set_previous(prev)
    assert np.array_equal(d.read_field(N.FIELD_PREVIOUS), prev)
    assert np.array_equal(d.positions(), s.position)
    bad = prev.copy()
    bad[5, 1] = np.nan
    with pytest.raises(N.VxError):
        d.set_previous(bad)
    d.close()


@pytest.mark.parametrize("count", [0, 1])
def test_contact_on_empty_and_single_rev_scenes(ctx, count):
    s = S.from_cells(np.zeros((count, 3), np.int32), M.component_id("iron"), M.table())
    d = N.DeviceScene(ctx, s)
    st = d.contact_project()
    assert st["candidates"] == 0 and st["pairs"] == 0 and st["contacts"] == 0
    assert len(d.contacts()) == 0
    assert d.resolve_contact_velocities(0.1, 0.35) == (0.0, 0.0)
    d.close()


def _loose(count):
    """count unbonded iron REVs in a row along x."""
    cells = np.zeros((count, 3), np.int32)
    cells[:, 0] = 2 * np.arange(count)
    s = S.from_cells(cells, M.component_id("iron"), M.table())
    s.neighbor[:] = S.EMPTY
    return s


def test_position_outside_the_bin_key_range_is_reported(ctx):
    s = _loose(2)
    d = N.DeviceScene(ctx, s)
    far = s.position.copy()
    far[1, 0] = 2.0e4  # 2e6 cells: beyond the 2^20 cells of a scene's bin keys
    d.set_positions(far)
    d.set_previous(far)
    with pytest.raises(N.VxError) as e:
        d.contact_project()
    assert e.value.status == N.VX_NONFINITE
    d.set_positions(s.position)  # the scene stays usable
    d.set_previous(s.position)
    st = d.contact_project()  # two cells apart: a candidate pair, no contact
    assert st["candidates"] == 1 and st["contacts"] == 0
    d.close()


def test_sweep_beyond_the_volume_limit_is_reported(ctx):
    s = _loose(2)
    d = N.DeviceScene(ctx, s)
    pos = s.position.copy()
    pos[0] += 3.0  # 302^3 bins, above the 2^24 one REV may sweep
    d.set_positions(pos)
    d.set_previous(s.position)
    with pytest.raises(N.VxError) as e:
        d.contact_project()
    assert e.value.status == N.VX_BAD_INPUT
    d.close()


def test_sweeps_beyond_the_total_volume_limit_are_reported(ctx):
    s = _loose(20)
    d = N.DeviceScene(ctx, s)
    pos = s.position + 2.5  # 252^3 bins each, under the per-REV limit; 20 of them above 2^28
    d.set_positions(pos)
    d.set_previous(s.position)
    with pytest.raises(N.VxError) as e:
        d.contact_project()
    assert e.value.status == N.VX_BAD_INPUT
    assert "together" in str(e.value)
    d.close()


def test_rotated_continuum_has_no_internal_contacts(ctx):
    s = S.scene_new((3, 3, 3))
    c, sn = math.cos(0.37), math.sin(0.37)
    r = np.array([[c, -sn, 0], [sn, c, 0], [0, 0, 1]])
    pos = (s.position @ r.T).astype(np.float32).astype(np.float64)
    d, st, oc = _check_project(ctx, s, pos, pos.copy())
    assert st["contacts"] == 0 and st["pairs"] < st["candidates"]
    d.close()


def test_crack_and_remote_self_contact(ctx):
    s = S.scene_new((3, 2, 1))
    s.neighbor[0, 0] = S.EMPTY
    pos = s.position.copy()
    pos[1] = pos[0] + np.array([CELL * 0.5, 0, 0])
    d, st, oc = _check_project(ctx, s, pos, pos.copy())
    assert any(c["i"] == 0 and c["j"] == 1 for c in oc)
    d.close()


def test_moving_voxel_cannot_tunnel_through_fixed_voxel(ctx):
    s = S.scene_new((2, 1, 1))
    s.neighbor[0, 0] = S.EMPTY
    s.kinematic[1] = 1
    prev = s.position.copy()
    pos = prev.copy()
    pos[0, 0] += 3.0 * CELL
    d, st, oc = _check_project(ctx, s, pos, prev)
    p = d.positions()
    assert st["contacts"] > 0 and p[1, 0] - p[0, 0] >= CELL - 1e-6
    d.close()


def _rubble(seed, n_side=6, jitter=0.45, speed=0.3, kin_layer=True):
    """Unbonded REVs on a jittered grid: random offsets up to `jitter` cells
    and random previous positions up to `speed` cells away, so that pairs
    overlap, cross and chain."""
    rng = np.random.default_rng(seed)
    cells = S.grid_cells(n_side, n_side, n_side)
    kin = (cells[:, 2] == 0) if kin_layer else np.zeros(len(cells), bool)
    s = S.from_cells(cells, M.component_id("iron"), M.table(), kinematic=kin.astype(np.uint8))
    s.neighbor[:] = S.EMPTY
    pos = s.position + rng.uniform(-jitter, jitter, s.position.shape) * CELL
    prev = pos + rng.uniform(-speed, speed, s.position.shape) * CELL
    pos[kin] = s.position[kin]
    prev[kin] = s.position[kin]
    return s, pos, prev


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_rubble_projection_matches_the_oracle(ctx, seed):
    s, pos, prev = _rubble(seed)
    d, st, oc = _check_project(ctx, s, pos, prev)
    assert st["contacts"] > 50 and st["sweeps"] >= 2
    d.close()


def test_staging_overflow_writes_in_a_second_pass(ctx):
    # an unbonded 14^3 pile stores about 13 pairs per REV, more than the
    # initial staging list (n / 4 + 4096): the first generation writes its pairs
    # in a second pass, later ones fit the grown list
    s, pos, prev = _rubble(5, n_side=14, jitter=0.2, speed=0.1)
    d, st, oc = _check_project(ctx, s, pos, prev)
    assert st["stored"] > s.n // 4 + 4096 and st["sweeps"] >= 2
    d.close()


def test_targeted_axes_do_not_move(ctx):
    s, pos, prev = _rubble(4)
    tmask = np.zeros(s.n, np.uint8)
    tmask[::3] = 5  # x and z targeted on every third REV
    d, st, oc = _check_project(ctx, s, pos, prev, tmask)
    p = d.positions()
    assert np.array_equal(p[::3, 0], pos[::3, 0]) and np.array_equal(p[::3, 2], pos[::3, 2])
    d.close()


def test_fast_revs_take_the_large_box_path(ctx):
    """Swept boxes of more than 4 bins per axis: REVs that crossed 3-6 cells
    in the substep, through the others."""
    s, pos, prev = _rubble(5, jitter=0.2, speed=0.1)
    rng = np.random.default_rng(6)
    fast = rng.choice(np.nonzero(s.kinematic == 0)[0], 12, replace=False)
    prev[fast] = pos[fast] + rng.uniform(-6, 6, (len(fast), 3)) * CELL
    d, st, oc = _check_project(ctx, s, pos, prev)
    assert st["contacts"] > 0
    d.close()


def test_deep_overlaps_replay_with_a_wider_bound(ctx):
    """Pairs overlapping by half a cell: one correction moves a REV by about
    2.5 mm, more than the first movement bound, so the sweep is replayed."""
    s = S.from_cells(S.grid_cells(8, 1, 1), M.component_id("iron"), M.table())
    s.neighbor[:] = S.EMPTY
    pos = s.position.copy()
    pos[:, 0] = np.arange(8) * CELL * 0.5
    d, st, oc = _check_project(ctx, s, pos, pos.copy())
    assert st["redone"] > 0
    d.close()


def test_contact_velocities_match_the_oracle(ctx):
    s, pos, prev = _rubble(7)
    d, st, oc = _check_project(ctx, s, pos, prev)
    rng = np.random.default_rng(8)
    vel = rng.normal(0, 1.0, (s.n, 3))
    vel[s.kinematic == 1] = 0.0
    d.set_velocities(vel)
    rh, fh = d.resolve_contact_velocities(0.1, 0.35)
    ov, orh, ofh = O.resolve_velocities(vel, vel, s.kinematic, s.mass.astype(np.float64), oc, 0.1, 0.35)
    assert np.array_equal(d.velocities(), ov), np.max(np.abs(d.velocities() - ov))
    assert abs(rh - orh) <= 1e-12 * max(orh, 1e-30) and abs(fh - ofh) <= 1e-12 * max(ofh, 1e-30)
    assert orh > 0 and ofh > 0
    d.close()


def test_given_contact_restitution(ctx):
    """normal_restitution_loss_is_converted_to_voxel_heat (src/collision.rs:809-868)"""
    s = S.scene_new((2, 1, 1))
    s.neighbor[0, 0] = S.EMPTY
    d = N.DeviceScene(ctx, s)
    vel = np.array([[1.0, 0, 0], [-1.0, 0, 0]])
    d.set_velocities(vel)
    contacts = np.array([(0, 1, 1, 1)], dtype=O.CONTACT_DTYPE)
    d.set_contacts(contacts)
    rh, fh = d.resolve_contact_velocities(0.25, 0.0)
    ov, orh, ofh = O.resolve_velocities(vel, vel, s.kinematic, s.mass.astype(np.float64), contacts, 0.25, 0.0)
    v = d.velocities()
    assert np.array_equal(v, ov)
    assert abs(v[1, 0] - v[0, 0] - 0.5) < 1e-6
    assert rh == orh and fh == 0.0
    d.close()


def _block(nx=6, ny=5, nz=4):
    cells = S.grid_cells(nx, ny, nz)
    return S.from_cells(cells, M.component_id("iron"), M.table(), kinematic=(cells[:, 2] == 0)), cells


def test_step_with_contact_rests_the_block_on_its_floor(ctx):
    """The block stands on the kinematic layer (not bonded to it) instead of
    falling through it; positions, velocities and contact counts against the
    oracle's step with contact."""
    s, cells = _block()
    g = (0.0, 0.0, float(np.float32(-9.81)))
    o = O.OracleStepper(s, fixed_dt=1e-3, substeps=4, iterations=20000, solver_tolerance=1e-14,
                        corotation_tolerance=0.0, corotation_iterations=2, gravity=g, fracture=True, contact=True)
    d = N.DeviceScene(ctx, s)
    p = N.step_params(1e-3, substeps=4, corotation_iterations=2, corotation_tolerance=0.0, gravity=g,
                      tolerance=1e-14, max_iterations=20000, precision=N.PRECISION_FP64, reuse=True,
                      fracture=True, contact=True)
    contacts = 0
    for _ in range(5):
        o.step()
        st = d.step(p)
        contacts += st["contacts"]
    assert contacts == o.d.contacts > 0
    dz = d.positions()[:, 2] - s.position[:, 2]
    assert np.max(np.abs(dz)) < 1e-5  # free fall would have dropped 1.2e-4 m
    disp = o.positions - s.position
    rel = np.linalg.norm(d.positions() - o.positions) / np.linalg.norm(disp)
    assert rel < 1e-8, rel
    v_scale = np.linalg.norm(disp) / 5e-3
    assert np.linalg.norm(d.velocities() - o.velocity.reshape(-1, 3)) < 1e-6 * v_scale
    d.close()


def test_step_keeps_unbonded_revs_apart(ctx):
    """unbonded_voxels_cannot_tunnel_through_each_other (src/collision.rs:870-898)
    through the device step."""
    s = S.scene_new((2, 1, 1))
    s.neighbor[0, 0] = S.EMPTY
    s.velocity[0] = (20.0, 0, 0)
    s.velocity[1] = (-20.0, 0, 0)
    d = N.DeviceScene(ctx, s)
    d.set_velocities(s.velocity)
    p = N.step_params(float(np.float32(0.001)), substeps=1, corotation_iterations=1, tolerance=1e-5,
                      max_iterations=20, precision=N.PRECISION_FP64, contact=True)
    d.step(p)
    x, v = d.positions(), d.velocities()
    assert x[1, 0] - x[0, 0] >= CELL - 1e-5
    assert (v[1] - v[0])[0] >= -1e-4
    d.close()


def test_pool_projects_every_slot_on_its_own(ctx):
    """Three rubble scenes at overlapping coordinates in one pool: each selected
    slot's projection is the oracle's projection of that scene alone (pairs
    never join two slots, the tile padding takes no part), and the slot left
    out of the call is untouched."""
    cases = [_rubble(11), _rubble(12, n_side=5), _rubble(13, jitter=0.2, speed=0.1)]
    pool = N.DevicePool(ctx, 8192, 4)
    slots = []
    for s, pos, prev in cases:
        k = pool.add(s)
        pool.set_positions(k, pos)
        pool.set_previous(k, prev)
        slots.append(k)
    st, per = pool.contact_project(enabled=slots[:2])
    pairs = 0
    for (s, pos, prev), k in zip(cases[:2], slots[:2]):
        op, oq, oc, ost = O.contact_project(pos, prev, s.position, s.kinematic, s.mass.astype(np.float64),
                                            s.neighbor)
        assert np.array_equal(pool.positions(k), op)
        assert np.array_equal(pool.previous(k), oq)
        assert per[k] == len(oc) > 0
        pairs += ost["pairs"]
    assert st["pairs"] == pairs and st["contacts"] == per[slots[0]] + per[slots[1]]
    s, pos, prev = cases[2]
    assert np.array_equal(pool.positions(slots[2]), pos) and np.array_equal(pool.previous(slots[2]), prev)
    assert per[slots[2]] == 0
    pool.close()


def test_pool_step_with_contact_matches_single_scene_steps(ctx):
    """vx_pool_step with the contact stage against vx_scene_step on each scene:
    two blocks resting on their floors and a free pair flying apart, three
    steps; both solve every pass to 1e-10, so positions agree to the solve
    error and the contact counts are equal."""
    sc = [_block()[0], _block(5, 4, 6)[0], S.scene_new((2, 1, 1))]
    sc[2].neighbor[0, 0] = S.EMPTY
    g = (0.0, 0.0, float(np.float32(-9.81)))
    p = N.step_params(1e-3, substeps=2, corotation_iterations=2, corotation_tolerance=0.0, gravity=g,
                      tolerance=1e-10, max_iterations=20000, precision=N.PRECISION_MIXED, fracture=True,
                      contact=True)
    pool = N.DevicePool(ctx, 16384, 4)
    slots = [pool.add(s) for s in sc]
    pool.set_velocities(slots[2], np.array([[20.0, 0, 0], [-20.0, 0, 0]]))
    counts = np.zeros(len(sc), np.int64)
    for _ in range(3):
        status, stats = pool.step(p)
        assert status == N.VX_OK
        counts += [stats[k]["contacts"] for k in slots]
    for idx, (s, k) in enumerate(zip(sc, slots)):
        d = N.DeviceScene(ctx, s)
        if idx == 2:
            d.set_velocities(np.array([[20.0, 0, 0], [-20.0, 0, 0]]))
        c = 0
        for _ in range(3):
            st = d.step(p)
            assert st["status"] == N.VX_OK
            c += st["contacts"]
        assert c == counts[idx] > 0
        x0 = s.position
        assert np.linalg.norm(pool.positions(k) - d.positions()) <= 1e-6 * max(np.linalg.norm(d.positions() - x0), 1e-9)
        d.close()
    x = pool.positions(slots[2])
    assert x[1, 0] - x[0, 0] >= CELL - 1e-5
    pool.close()
