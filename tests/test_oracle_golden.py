"""Pins the CPU oracle to the reference's own unit tests and probes.

Each test restates one reference test (cited) with its inputs and its stated
tolerance, run against the oracle restatement. These fix the oracle's results
to the precision the reference itself asserts.
"""
import math

import numpy as np
import pytest

import pyoracle as O
from vxsim import materials as M
from vxsim import scenes as S

AREA32 = np.float32(np.float32(0.01) * np.float32(0.01))
CELL32 = np.float32(0.01)


def wood_chop_scene():
    """`scene()` of src/solver.rs:885-892: wood_chop.ron with 2x2x2 trunk and 2x2x1 ground."""
    return S.scene_new((2, 2, 2), ground=(2, 2, 1), anisotropy=1.0)


def quat_from_rotation_z(angle):
    return np.array([0.0, 0.0, math.sin(angle / 2), math.cos(angle / 2)])


def rotate(q, v):
    x, y, z, w = q
    b = np.array([x, y, z])
    return v * (w * w - b @ b) + b * (2 * v @ b) + np.cross(b, v) * (2 * w)


# -- src/solver.rs:1033-1060 -------------------------------------------------
def test_actual_vertical_wood_bonds_are_stronger_than_horizontal_bonds():
    s = wood_chop_scene()
    o = O.OracleScene(s)
    i = 0
    vj = int(s.neighbor[2, i])
    hj = int(s.neighbor[0, i])
    assert vj != S.EMPTY and hj != S.EMPTY
    v = o.bond_limits(i, vj, [0, 0, 1])
    h = o.bond_limits(i, hj, [1, 0, 0])
    assert v.tension >= h.tension * 39.0
    assert v.compression >= h.compression * 24.0
    assert v.shear >= h.shear * 3.9
    assert abs(v.tension - 100e6) < 1.0
    assert abs(h.tension - 2.5e6) < 1.0
    assert abs(v.compression - 50e6) < 1.0
    assert abs(h.compression - 2e6) < 1.0
    assert abs(v.shear - 12e6) < 1.0
    assert abs(h.shear - 3e6) < 1.0
    vk = o.stiffness_matrix(i, vj, O.basis(2, [0, 0, 0, 1]))[0, 0]
    hk = o.stiffness_matrix(i, hj, O.basis(0, [0, 0, 0, 1]))[0, 0]
    assert vk > hk * 15.0


# -- src/solver.rs:1023-1031 -------------------------------------------------
def test_stiffness_has_shear_and_is_symmetric():
    s = wood_chop_scene()
    o = O.OracleScene(s)
    k = o.stiffness_matrix(0, 1, np.eye(3))
    assert k[1, 1] > 0 and k[2, 2] > 0 and np.linalg.det(k) > 0
    assert np.all(np.abs(k - k.T) < 1e-3)


# -- src/solver.rs:1009-1021 -------------------------------------------------
def test_rest_and_rigid_rotation_have_no_strain():
    s = wood_chop_scene()
    q = quat_from_rotation_z(0.7)
    s.position = np.array([rotate(q, p) for p in s.position])
    o = O.OracleScene(s)
    o.fit_rotations()
    rot = o.rotations()
    frame = O.basis(0, rot[0])
    j = int(s.neighbor[0, 0])
    pos = o.positions()
    c = frame.T @ (pos[j] - pos[0]) - np.array([1.0, 0, 0]) * O.VXO_CELL
    assert np.linalg.norm(c) < 1e-6


def test_fit_rotations_recovers_a_rigid_rotation_and_reports_the_angle():
    s = S.from_cells(S.grid_cells(3, 3, 3), 1, M.table(), anisotropy=1.0)
    q = np.array([0.1, -0.2, 0.3, 0.9])
    q /= np.linalg.norm(q)
    centre = s.position.mean(axis=0)
    s.position = np.array([centre + rotate(q, p - centre) for p in s.position])
    o = O.OracleScene(s)
    angle = o.fit_rotations()
    rot = o.rotations()
    assert np.all(np.abs(np.abs(rot @ q) - 1.0) < 1e-12)
    assert abs(angle - 2 * math.acos(abs(q[3]))) < 1e-9


# -- src/solver.rs:1112-1161 -------------------------------------------------
def test_heated_bond_rest_length_follows_thermal_expansion():
    from dataclasses import replace
    t = M.table()
    iron = M.component_id("iron")
    t[iron] = replace(t[iron], thermal_expansion_parallel=1e-5, thermal_expansion_perpendicular=1e-5)
    s = S.from_cells([[0, 0, 0], [1, 0, 0]], iron, t)
    s.thermal_delta[:] = 393.15 - 293.15
    s.fix_voxels([0])
    o = O.OracleScene(s)
    frame, mk, k, rest = o.make_constraint(0, 0, 1)
    assert abs(rest[0] / O.VXO_CELL - 1.001) < 1e-6


def test_thermal_expansion_projects_parallel_and_transverse_fiber_coefficients():
    t = M.table()
    cells = [[-1, 0, 0], [0, 0, 0], [1, 0, 0], [4, 0, 0], [4, 0, 1], [4, 0, 2]]
    s = S.from_cells(cells, 1, t, anisotropy=1.0)
    s.thermal_delta[:] = 393.15 - 293.15
    o = O.OracleScene(s)
    transverse = o.bond_thermal_rest(1, 2, O.basis(0, [0, 0, 0, 1]))[0]
    parallel = o.bond_thermal_rest(4, 5, O.basis(2, [0, 0, 0, 1]))[0]
    assert abs(transverse / O.VXO_CELL - 1.003) < 1e-6
    assert abs(parallel / O.VXO_CELL - 1.0003) < 1e-6
    assert transverse > parallel * 1.002


# -- src/fracture.rs:310-549 -------------------------------------------------
def k_of(m):
    d = np.array([m.young, m.shear, m.shear], np.float32) * AREA32 / CELL32
    return np.diag(d.astype(np.float64))


def test_brittle_failure_has_no_plasticity():
    m = M.table()[3]
    b = O.VxoBond(neighbor=1)
    lim = O.pair_limits(m, m, [1.0, 1.0], [0.0, 0.0])
    u = np.array([1.1 * np.float32(m.tensile_strength) / np.float32(m.young) * CELL32, 0, 0])
    O.fracture_update(b, u, k_of(m), lim, 0.001, O.default_fracture_config())
    assert b.neighbor == S.EMPTY
    assert list(b.plastic) == [0.0, 0.0, 0.0]


def test_metal_yields_heats_and_only_then_tears():
    m = M.table()[2]
    b = O.VxoBond(neighbor=1)
    lim = O.pair_limits(m, m, [1.0, 1.0], [0.0, 0.0])
    heat = 0.0
    for n in range(1, 301):
        d = O.fracture_update(b, np.array([n * 0.001 * 0.01, 0, 0]), k_of(m), lim, 0.001,
                              O.default_fracture_config())
        heat += d.plastic_heat
        if n == 2:
            assert b.neighbor != S.EMPTY
            assert b.equivalent_plastic_strain > 0.0
        if b.neighbor == S.EMPTY:
            break
    assert b.neighbor == S.EMPTY
    assert heat > 0.0
    assert b.equivalent_plastic_strain > 0.1


def test_energy_removed_is_not_duplicated():
    m = M.table()[3]
    b = O.VxoBond(neighbor=1)
    u = np.array([2.0 * m.tensile_strength / m.young * 0.01, 0, 0])
    k = k_of(m)
    before = 0.5 * u @ (k @ u)
    d = O.fracture_update(b, u, k, O.pair_limits(m, m, [1.0, 1.0], [0.0, 0.0]), 0.001,
                          O.default_fracture_config())
    assert abs(d.total() - before) < 1e-8


def test_sustained_subcritical_load_does_not_count_as_cycles():
    b = O.VxoBond(neighbor=1)
    c = O.default_fracture_config()
    for _ in range(10000):
        O.fatigue(b, 0.8, c)
    assert b.fatigue_damage == 0.0


def test_cyclic_subcritical_load_accumulates_damage():
    b = O.VxoBond(neighbor=1)
    c = O.default_fracture_config()
    c.fatigue_cycles = 10.0
    c.fatigue_exponent = 1.0
    for _ in range(50):
        O.fatigue(b, 0.8, c)
        O.fatigue(b, -0.8, c)
    assert b.fatigue_damage == 1.0


def test_cyclic_subcritical_stress_breaks_bond_through_constitutive_update():
    m = M.table()[2]
    limits = O.pair_limits(m, m, [1.0, 1.0], [0.0, 0.0])
    b = O.VxoBond(neighbor=1)
    c = O.default_fracture_config()
    c.fatigue_cycles = 2.0
    c.fatigue_exponent = 1.0
    c.fatigue_threshold = 0.1
    amplitude = 0.4 * m.tensile_strength / m.young * 0.01
    k = k_of(m)
    for _ in range(100):
        r = O.fracture_update(b, np.array([amplitude, 0, 0]), k, limits, 0.001, c)
        assert b.neighbor == 1
        assert b.fatigue_damage == 0.0
        assert r.total() == 0.0
    dissipated = 0.0
    failure = None
    for _ in range(20):
        for sign in (-1.0, 1.0):
            r = O.fracture_update(b, np.array([sign * amplitude, 0, 0]), k, limits, 0.001, c)
            dissipated += r.total()
            if b.neighbor == S.EMPTY:
                failure = r
                break
        if b.neighbor == S.EMPTY:
            break
    assert b.neighbor == S.EMPTY
    assert b.damage == 1.0
    assert b.fatigue_damage == 1.0
    assert dissipated > 0.0
    u = np.array([amplitude, 0, 0])
    released = 0.5 * u @ (k @ u)
    assert abs(failure.total() - released) <= released * 1e-6


def test_wood_has_tension_and_compression_anisotropy():
    m = M.table()[1]
    along = O.pair_limits(m, m, [1.0, 1.0], [1.0, 1.0])
    across = O.pair_limits(m, m, [0.0, 0.0], [1.0, 1.0])
    assert along.tension / across.tension >= 10.0
    assert along.compression / across.compression >= 10.0
    assert across.ductility == 0.0
    assert along.ductility == 1.0


def test_wood_fracture_energy_follows_bond_alignment():
    m = M.table()[1]
    assert O.pair_limits(m, m, [1.0, 1.0], [1.0, 1.0]).fracture_energy == 350.0
    assert O.pair_limits(m, m, [0.0, 0.0], [1.0, 1.0]).fracture_energy == 80.0
    assert O.pair_limits(m, m, [0.5, 0.5], [1.0, 1.0]).fracture_energy == 215.0
    assert O.pair_limits(m, m, [0.0, 0.0], [0.0, 0.0]).fracture_energy == 350.0


def test_mixed_wood_shear_failure_does_not_wait_for_higher_yield_stress():
    m = M.table()[1]
    b = O.VxoBond(neighbor=1)
    limits = O.pair_limits(m, m, [0.5, 0.5], [1.0, 1.0])
    assert limits.ductility > 0.0
    shear_strain = 1.1 * limits.shear / m.shear * 0.01
    O.fracture_update(b, np.array([0, shear_strain, 0]), k_of(m), limits, 0.001, O.default_fracture_config())
    assert b.equivalent_plastic_strain == 0.0
    assert b.damage > 0.0
    assert b.neighbor == 1


# -- validation/cuda_sparse_probe.py:268-343 (analytic 2-node PCG) ----------
def two_node_rows():
    e = S.EMPTY
    rhs = np.array([1.0, 2.0, 3.0, 4.0, -1.0, 0.5], np.float32)
    diag = np.array([2.0, 0, 0, 0, 2.0, 0, 0, 0, 2.0] * 2, np.float32)
    inv = np.array([0.5, 0, 0, 0, 0.5, 0, 0, 0, 0.5] * 2, np.float32)
    nbr = np.array([1, e, e, e, e, e, e, 0, e, e, e, e], np.uint32)
    blocks = np.zeros(108, np.float32)
    for node, edge in ((0, 0), (1, 1)):
        base = node * 54 + edge * 9
        for a in range(3):
            blocks[base + a * 3 + a] = -0.2
    return dict(n=2, rhs=rhs, nbr6=nbr, diag9=diag, blocks54=blocks, inv9=inv)


def two_node_expected():
    b = two_node_rows()["rhs"].astype(np.float64)
    x = np.zeros(6)
    for c in range(3):
        b0, b1 = b[c], b[3 + c]
        x[c] = (2.0 * b0 + 0.2 * b1) / 3.96
        x[3 + c] = (0.2 * b0 + 2.0 * b1) / 3.96
    return x.reshape(2, 3)


def test_analytic_two_node_pcg_cuda_sequence():
    st, dx, it, res = O.cuda_pcg_emulate(two_node_rows(), 80, 1e-5)
    assert st == 0
    assert np.max(np.abs(dx - two_node_expected())) <= 1e-5
    assert res <= 1e-5


def test_analytic_two_node_pcg_cpu_loop():
    dx, it, res = O.pcg_rows_f32(two_node_rows(), 80, 1e-5)
    assert np.max(np.abs(dx - two_node_expected())) <= 1e-5


# -- src/solver.rs:1175-1205 -------------------------------------------------
def test_coupled_solve_has_uniform_axial_traction():
    s = S.scene_new((10, 2, 2), anisotropy=1.0)
    n = s.n
    mask = np.zeros(n, np.uint8)
    target = np.zeros((n, 3))
    for i in range(n):
        if i % 10 == 0:
            mask[i] = 7
            target[i] = s.position[i]
        if i % 10 == 9:
            mask[i] = 7
            target[i] = s.position[i] + np.array([0.00002, 0, 0])
    st = O.OracleStepper(s, fixed_dt=0.001, substeps=1, iterations=100, corotation_iterations=4)
    st.set_targets(mask, target)
    st.step()
    f = st.last_forces()[0]
    bonded = st.o.nbr.reshape(3, n)[0] != S.EMPTY
    forces = f[bonded, 0]
    assert forces.min() > 0 and forces.max() / forces.min() < 1.02, (forces.min(), forces.max())
    assert st.broken == 0


# -- src/solver.rs:1163-1173 -------------------------------------------------
def test_equilibrium_does_not_break():
    s = wood_chop_scene()
    initial = s.position.copy()
    st = O.OracleStepper(s, fixed_dt=0.016666668, substeps=4, iterations=40, corotation_iterations=4)
    st.step()
    assert st.broken == 0
    assert np.all(np.linalg.norm(st.positions - initial, axis=1) < 1e-6)


# -- tests/cpu_preconditioners.rs:8-79 --------------------------------------
def loaded_iron_lattice():
    iron = M.component_id("iron")
    cells = [[x, y, z] for x in range(3) for y in range(2) for z in range(2)]
    s = S.from_cells(cells, iron, M.table())
    s.fix_voxels([0, 1, 2, 3])
    s.target_mask[7] = 1
    s.target[7, 0] = s.position[7, 0]
    s.loads[11] = [0.0, 3000.0, 2000.0]
    return s


@pytest.mark.parametrize("tolerance", [1e-5, 1e-12])
def test_block_jacobi_partially_constrained_scene(tolerance):
    s = loaded_iron_lattice()
    start = s.position[11].copy()
    fixed_x = s.position[7, 0]
    st = O.OracleStepper(s, fixed_dt=0.001, substeps=1, iterations=256, solver_tolerance=tolerance)
    st.set_targets(s.target_mask, s.target)
    for _ in range(8):
        st.step()
        assert np.all(np.isfinite(st.positions))
        assert st.d.solver_residual <= max(tolerance, 1e-5)
        assert st.positions[7, 0] == fixed_x
    assert np.linalg.norm(st.positions[11] - start) > 0.0


def test_block_jacobi_tolerance_agreement_matches_reference_bound():
    out = []
    for tol in (1e-5, 1e-12):
        s = loaded_iron_lattice()
        st = O.OracleStepper(s, fixed_dt=0.001, substeps=1, iterations=256, solver_tolerance=tol)
        st.set_targets(s.target_mask, s.target)
        for _ in range(8):
            st.step()
        out.append(st.positions.copy())
    assert np.max(np.linalg.norm(out[0] - out[1], axis=1)) < 2e-5


# -- oracle self-consistency -------------------------------------------------
def test_fp64_pcg_converges_to_true_residual_on_wood_cube():
    s = S.wood_cube()
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    o.factor_block_jacobi()
    dx, it, res = o.pcg(5000, 1e-12)
    assert res < 1e-12
    assert o.true_residual(dx) < 1e-11
    # the f32 restatement of the reference's CPU loop reaches its own tolerance
    rows = o.pack_rows()
    dx32, it32, res32 = O.pcg_rows_f32(rows, 2000, 1e-5)
    assert res32 < 1e-5
    ref = dx[rows["active"]]
    assert np.linalg.norm(dx32 - ref) / np.linalg.norm(ref) < 1e-3


def test_topology_matches_dense_lattice_rule():
    rng = np.random.default_rng(0)
    cells = S.grid_cells(6, 5, 4)
    keep = rng.random(len(cells)) < 0.7
    cells = cells[keep]
    kin = (rng.random(len(cells)) < 0.2).astype(np.uint8)
    nbr_py = S.build_topology(cells, kin)
    nbr_c = np.zeros(3 * len(cells), np.uint32)
    O.lib().vxo_build_topology(O.ptr(np.ascontiguousarray(cells, np.int32), O.C.c_int32),
                               O.ptr(kin, O.C.c_uint8), len(cells), O.ptr(nbr_c, O.C.c_uint32))
    assert np.array_equal(nbr_py.reshape(-1), nbr_c)


def test_cluster_numbering_follows_the_reference_test():
    """connecting_adjacent_revs_rebuilds_topology_and_accepts_either_order
    (src/scene.rs:2082-2103): a fixed and a free iron REV are not bonded (one
    cluster); once released there are two; bonded, one again."""
    empty = np.full(6, 0xFFFFFFFF, np.uint32)
    cl, cnt = O.rebuild_clusters(empty, np.array([1, 0], np.uint8))
    assert cnt == 1 and list(cl) == [0xFFFFFFFF, 0]
    cl, cnt = O.rebuild_clusters(empty, np.array([0, 0], np.uint8))
    assert cnt == 2 and list(cl) == [0, 1]
    bonded = empty.copy()
    bonded[0] = 1  # bonds[0][0].neighbor = 1
    cl, cnt = O.rebuild_clusters(bonded, np.array([0, 0], np.uint8))
    assert cnt == 1 and list(cl) == [0, 0]


def test_cluster_ids_agree_with_a_breadth_first_restatement():
    """On a lattice with 60% of its bonds removed, the union-find numbering
    equals components found by breadth-first search, numbered by first
    non-kinematic REV."""
    rng = np.random.default_rng(3)
    s = S.wood_cube(8)
    nb = s.neighbor.copy()
    nb[rng.random(nb.shape) < 0.6] = 0xFFFFFFFF
    n = s.n
    adj = [[] for _ in range(n)]
    for a in range(3):
        for i in range(n):
            j = int(nb[a, i])
            if j != 0xFFFFFFFF:
                adj[i].append(j)
                adj[j].append(i)
    comp = [-1] * n
    for i in range(n):
        if comp[i] < 0:
            comp[i], todo = i, [i]
            while todo:
                x = todo.pop()
                for y in adj[x]:
                    if comp[y] < 0:
                        comp[y] = i
                        todo.append(y)
    ids, want = {}, []
    for i in range(n):
        if s.kinematic[i]:
            want.append(0xFFFFFFFF)
        else:
            want.append(ids.setdefault(comp[i], len(ids)))
    cl, cnt = O.rebuild_clusters(nb, s.kinematic)
    assert list(cl) == want and cnt == len(ids) and cnt > 5
