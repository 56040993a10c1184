"""The oracle's contact restatement (collision::project and
resolve_velocities_with_precontact, src/collision.rs) against the reference's
own collision tests (src/collision.rs:672-1016), restated. Scenes follow
Scene::new with scenes/wood_chop.ron's settings where the reference loads it
(corotation_iterations 4, iterations 40, restitution 0.1, friction 0.35).
CPU only."""
import math

import numpy as np
import pytest

import pyoracle as O
from vxsim import materials as M
from vxsim import scenes as S

CELL = float(np.float32(0.01))


def _pair_scene(break_bond=True):
    s = S.scene_new((2, 1, 1))
    if break_bond:
        s.neighbor[0, 0] = S.EMPTY
    return s


def _project(s, pos, prev, target_mask=None):
    return O.contact_project(pos, prev, s.position, s.kinematic, s.mass.astype(np.float64), s.neighbor,
                             target_mask)


def test_rigidly_rotated_continuum_has_no_internal_box_contacts():
    s = S.scene_new((3, 3, 3))
    c, sn = math.cos(0.37), math.sin(0.37)
    r = np.array([[c, -sn, 0], [sn, c, 0], [0, 0, 1]])
    pos = (s.position @ r.T).astype(np.float32).astype(np.float64)
    p, q, contacts, st = _project(s, pos, pos.copy())
    assert len(contacts) == 0
    assert np.array_equal(p, pos) and np.array_equal(q, pos)
    assert st["candidates"] > st["pairs"] > 0  # the local continuum pairs were filtered


def test_local_exclusion_does_not_hide_a_crack_or_remote_self_contact():
    s = S.scene_new((3, 2, 1))
    adj = _adjacency(s.neighbor)
    rest = s.position.astype(np.float32).astype(np.float64).reshape(-1).copy()
    local = lambda a, i, j: O.lib().vxo_local_continuum_pair(O.ptr(rest, O.C.c_double), O.ptr(a, O.C.c_uint32), i, j)
    assert local(adj, 0, 4)
    assert not local(adj, 0, 2)
    s.neighbor[0, 0] = S.EMPTY
    adj = _adjacency(s.neighbor)
    assert not local(adj, 0, 1)
    pos = s.position.copy()
    pos[1] = pos[0] + np.array([CELL * 0.5, 0, 0])
    _, _, contacts, _ = _project(s, pos, pos.copy())
    assert any(c["i"] == 0 and c["j"] == 1 for c in contacts)


def _adjacency(neighbor):
    n = neighbor.shape[1]
    adj = np.full((n, 6), S.EMPTY, np.uint32)
    for a in range(3):
        for i in range(n):
            j = neighbor[a, i]
            if j != S.EMPTY:
                adj[i, 2 * a + 1] = j
                adj[j, 2 * a] = i
    return np.ascontiguousarray(adj.reshape(-1))


def test_moving_voxel_cannot_tunnel_through_fixed_voxel():
    s = _pair_scene()
    s.kinematic[1] = 1
    pos = s.position.copy()
    prev = pos.copy()
    wall = pos[1].copy()
    pos[0, 0] += 3.0 * CELL
    p, _, contacts, _ = _project(s, pos, prev)
    assert len(contacts) > 0
    assert np.array_equal(p[1], wall)
    assert wall[0] - p[0, 0] >= CELL - 1e-6


def test_sliding_contact_dissipates_tangent_energy_into_voxel_heat():
    s = _pair_scene()
    s.kinematic[1] = 1
    pos = s.position.copy()
    prev = pos.copy()
    vel = np.zeros((2, 3))
    vel[0] = (1.0, 2.0, 5.0)
    pos[0, 0] += CELL * 0.2
    tmask = np.array([4, 0], np.uint8)  # REV 0's z axis targeted
    p, _, contacts, _ = _project(s, pos, prev, tmask)
    assert any(c["i"] == 0 and c["j"] == 1 for c in contacts)
    mass = float(s.mass[0])
    ke_before = 0.5 * mass * vel[0, 1] ** 2
    v, rh, fh = O.resolve_velocities(vel, vel, s.kinematic, s.mass.astype(np.float64), contacts, 0.1, 0.35, tmask)
    dissipated = ke_before - 0.5 * mass * v[0, 1] ** 2
    assert abs(v[0, 1]) < 2.0
    assert v[0, 2] == 5.0
    assert dissipated > 0.0
    assert abs(dissipated - fh) < 1e-7


def test_normal_restitution_loss_is_converted_to_voxel_heat():
    s = _pair_scene()
    m = s.mass.astype(np.float64)
    vel = np.array([[1.0, 0, 0], [-1.0, 0, 0]])
    contacts = np.array([(0, 1, 1, 1)], dtype=O.CONTACT_DTYPE)
    v, rh, fh = O.resolve_velocities(vel, vel, s.kinematic, m, contacts, 0.25, 0.0)
    p0, p1 = (m[:, None] * vel).sum(0), (m[:, None] * v).sum(0)
    ke = lambda u: float((0.5 * m * (u ** 2).sum(1)).sum())
    assert np.linalg.norm(p1 - p0) < 1e-6
    assert abs(v[1, 0] - v[0, 0] - 0.5) < 1e-6
    dissipated = ke(vel) - ke(v)
    assert dissipated > 0.0
    assert abs(dissipated - rh) < 1e-8
    assert fh == 0.0


def test_touching_contact_persists_after_projection_slop():
    iron = M.component_id("iron")
    cells = np.array([[0, 0, 0], [1, 0, 0]], np.int32)
    s = S.from_cells(cells, iron, M.table(), kinematic=np.array([1, 0], np.uint8))
    s.kinematic[0] = 0  # release_voxel: no bond forms (the flags differed at creation)
    assert np.all(s.neighbor == S.EMPTY)
    pos = s.position.copy()
    pos[1, 0] += 0.005
    prev = pos.copy()
    vel = np.array([[0.01, 0, 0], [-0.01, 0, 0]])
    pos[0, 0] += 0.002503
    pos[1, 0] -= 0.002503
    m = s.mass.astype(np.float64)
    p, q, impact, _ = _project(s, pos, prev)
    assert len(impact) == 1 and impact[0]["new_impact"]
    v, _, _ = O.resolve_velocities(vel, vel, s.kinematic, m, impact, 0.1, 0.35)
    p2, _, resting, _ = _project(s, p, p.copy())
    assert len(resting) == 1 and not resting[0]["new_impact"]
    assert np.linalg.norm(p2[1] - p2[0]) <= CELL + 2e-6


def _stepper(s, **kw):
    cfg = dict(fixed_dt=float(np.float32(0.001)), substeps=4, iterations=40, solver_tolerance=1e-5,
               corotation_tolerance=1e-5, corotation_iterations=4, gravity=(0.0, 0.0, 0.0), contact=True)
    cfg.update(kw)
    return O.OracleStepper(s, **cfg)


def test_free_fall_has_no_invisible_ground():
    s = S.scene_new((1, 1, 1))
    start = s.position[0, 2]
    o = _stepper(s, substeps=1, gravity=(0.0, 0.0, float(np.float32(-9.81))))
    for _ in range(100):
        o.step()
    expected = start - 9.81 * 0.001 * 0.001 * 5050.0
    assert abs(o.positions[0, 2] - expected) < 2e-6
    assert o.positions[0, 2] < 0.0


def test_unbonded_voxels_cannot_tunnel_through_each_other():
    s = _pair_scene()
    s.velocity[0] = (20.0, 0, 0)
    s.velocity[1] = (-20.0, 0, 0)
    o = _stepper(s, substeps=1, iterations=20, corotation_iterations=1)
    o.step()
    p = o.positions
    v = o.velocity.reshape(-1, 3)
    assert p[1, 0] - p[0, 0] >= CELL - 1e-5
    assert (v[1] - v[0])[0] >= -1e-4


def test_initially_overlapping_voxels_are_projected_to_touching():
    s = _pair_scene()
    mid = (s.position[0] + s.position[1]) * 0.5
    s.position[0] = mid
    s.position[1] = mid
    o = _stepper(s, substeps=1, iterations=20, corotation_iterations=1, rest=S.scene_new((2, 1, 1)).position)
    o.step()
    p = o.positions
    assert p[1, 0] - p[0, 0] >= CELL - 1e-5


def test_resting_contact_under_compression_does_not_accumulate_impact_heat():
    s = _pair_scene()
    s.loads[0] = (0.1, 0, 0)
    s.loads[1] = (-0.1, 0, 0)
    o = _stepper(s, fixed_dt=float(np.float32(0.01)), substeps=2, iterations=1, corotation_iterations=1,
                 restitution=0.0, friction=0.0)
    for _ in range(20):
        o.step()
    p = o.positions
    assert np.linalg.norm(p[1] - p[0]) <= CELL + 2e-6
    assert o.d.restitution_heat == 0.0
    assert o.d.contacts > 0


def test_block_rests_on_its_kinematic_floor():
    """The capture's block (36 x 32 x 32 iron at reduced size 6 x 5 x 4): with
    contact the free layers stand on the kinematic bottom layer instead of
    falling through it."""
    cells = S.grid_cells(6, 5, 4)
    s = S.from_cells(cells, M.component_id("iron"), M.table(), kinematic=(cells[:, 2] == 0))
    o = _stepper(s, substeps=4, iterations=160, corotation_iterations=2, gravity=(0.0, 0.0, float(np.float32(-9.81))))
    for _ in range(5):
        o.step()
    dz = o.positions[:, 2] - s.position[:, 2]
    assert np.all(dz[cells[:, 2] == 0] == 0.0)
    assert np.max(np.abs(dz)) < 1e-5  # free fall would have dropped 1.2e-4 m
    assert o.d.contacts > 0
