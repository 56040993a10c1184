"""CUDA path vs the CPU oracle through the C ABI (needs a B200).

Bars: topology bit-exact; rotations and FP64 displacements within 1e-10
relative of the FP64 oracle; the FP32/FP64-refinement form within its stated
true-residual target of 1e-8 and its error against an FP64 solve to the FP64
floor reported; bond-stress ratios within 1e-9 relative; the compatibility
shim within the f32 tolerances of the reference's own CUDA probe.
"""
import math

import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def deformed(scene, seed=0, amp=2e-4, twist=0.3):
    """Rigidly rotate and randomly perturb REV positions (nontrivial rotations)."""
    rng = np.random.default_rng(seed)
    c = scene.position.mean(axis=0)
    th = twist
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    p = (scene.position - c) @ R.T + c
    p += rng.normal(0, amp, size=p.shape)
    scene.position = p
    scene.target = np.where((scene.target_mask[:, None] & np.array([1, 2, 4])) > 0, p, scene.target)
    return scene


# -- topology ------------------------------------------------------------------------
def test_topology_bit_exact(ctx):
    rng = np.random.default_rng(3)
    cells = S.grid_cells(17, 9, 11, origin=(-5, 3, -2))
    cells = cells[rng.random(len(cells)) < 0.8]
    cells = cells[rng.permutation(len(cells))]
    kin = (rng.random(len(cells)) < 0.15).astype(np.uint8)
    gpu = ctx.build_topology(cells, kin)
    assert np.array_equal(gpu, S.build_topology(cells, kin))


def test_topology_rejects_duplicates(ctx):
    cells = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 0]], np.int32)
    with pytest.raises(N.VxError) as e:
        ctx.build_topology(cells, np.zeros(3, np.uint8))
    assert e.value.status == N.VX_BAD_INPUT


# -- rotation fit ----------------------------------------------------------------------
def test_fit_rotations_matches_oracle(ctx):
    s = deformed(S.mixed_block(8, seed=4), seed=5, amp=5e-4, twist=0.4)
    o = O.OracleScene(s)
    ang_o = o.fit_rotations()
    d = N.DeviceScene(ctx, s)
    ang_g = d.fit_rotations()
    qo, qg = o.rotations(), d.rotations()
    dots = np.abs(np.sum(qo * qg, axis=1))
    assert np.max(np.abs(dots - 1.0)) < 1e-12
    assert abs(ang_g - ang_o) <= 1e-10 * max(ang_o, 1e-30)


# -- one FP64 pass ------------------------------------------------------------------------
def pass_pair(ctx, scene, h, tol, max_it, precision=N.PRECISION_FP64, fits=1):
    o = O.OracleScene(scene)
    d = N.DeviceScene(ctx, scene)
    for _ in range(fits):
        o.fit_rotations()
        d.fit_rotations()
    x0 = scene.position.copy()
    it_o, res_o = o.solve_coupled(h, max_it, tol)
    st = d.corotational_pass(h, tol, max_it, precision=precision)
    return o, d, x0, (it_o, res_o), st


def test_fp64_pass_fixed_iterations_track_oracle(ctx):
    """Same recurrences: after a fixed number of iterations the iterates agree."""
    s = deformed(S.mixed_block(10, seed=6), seed=7)
    o, d, x0, (it_o, _), st = pass_pair(ctx, s, 1e-3, 1e-300, 40)
    assert it_o == 40 and st["iterations"] == 40
    dx_o = o.positions() - x0
    dx_g = d.positions() - x0
    assert rel(dx_g, dx_o) < 1e-10


def loaded_wood_cube():
    """The 10^3 wood cube with its top layer lifted onto the +0.1 mm targets,
    as the substep's prediction leaves it before the pass (src/solver.rs:506-512)."""
    return S.impose_axis_targets(S.wood_cube())


def test_wood_cube_fp64_displacements_match_oracle(ctx):
    """10^3 wood cube under its +0.1 mm top-layer load, plain FP64, solved to the
    FP64 floor on both sides: the pass's correction dx (about 8.9e-5 m at most)
    agrees with the oracle's to 1e-10 relative. dx is taken against the
    positions the pass started from; their FP64 spacing near 0.09 m (1.4e-17 m)
    is 1.6e-13 of the largest correction, far below the bar."""
    s = loaded_wood_cube()
    o, d, x0, (it_o, res_o), st = pass_pair(ctx, s, 1e-3, 1e-13, 10000)
    dx_o = o.positions() - x0
    dx_g = d.positions() - x0
    # the load reaches the system: both sides move the REVs under the top layer
    assert 8.5e-5 < np.abs(dx_o).max() < 9.5e-5 and 8.5e-5 < np.abs(dx_g).max() < 9.5e-5
    err = rel(dx_g, dx_o)
    print(f"C1 loaded wood cube: |dx|max {np.abs(dx_g).max():.4e} m, {st['iterations']} / {it_o} iterations, "
          f"rel err vs oracle {err:.3e}")
    assert err < 1e-10
    assert st["true_residual"] < 1e-12
    assert abs(st["iterations"] - it_o) <= 2


def test_wood_cube_reference_tolerance(ctx):
    """At the workload's 1e-10 target both sides reach it on the loaded cube, and
    the corrections agree to the solve error (kappa times the tolerance)."""
    s = loaded_wood_cube()
    o, d, x0, (it_o, res_o), st = pass_pair(ctx, s, 1e-3, 1e-10, 10000)
    assert res_o < 1e-10 and st["residual"] < 1e-10 and st["converged"] == 1
    assert st["true_residual"] < 2e-10
    assert abs(st["iterations"] - it_o) <= 1
    assert np.abs(d.positions() - x0).max() > 8.5e-5
    assert rel(d.positions() - x0, o.positions() - x0) < 1e-8


def test_unloaded_wood_cube_stays_at_rest(ctx):
    """Without the targets imposed the cube is at rest: the right-hand side is
    rounding residue and neither side moves a REV by more than 1e-8 m."""
    s = S.wood_cube()
    o, d, x0, _, st = pass_pair(ctx, s, 1e-3, 1e-10, 10000)
    assert np.abs(o.positions() - x0).max() < 1e-8
    assert np.abs(d.positions() - x0).max() < 1e-8


def test_reused_preconditioner_matches_oracle(ctx):
    """Passes > 0 keep the pass-0 block-Jacobi factor (CPU path, src/solver.rs:554, :1639)."""
    s = deformed(S.mixed_block(8, seed=8), seed=9)
    o = O.OracleScene(s)
    d = N.DeviceScene(ctx, s)
    x0 = s.position.copy()
    for p in range(3):
        o.fit_rotations()
        d.fit_rotations()
        # the predicted positions stay those of the substep across passes (src/solver.rs:542)
        o.solve_coupled(1e-3, 25, 1e-300, reuse=p > 0, predicted=x0)
        d.corotational_pass(1e-3, 1e-300, 25, reuse=p > 0)
    assert rel(d.positions() - x0, o.positions() - x0) < 1e-9


# -- mixed precision ---------------------------------------------------------------------
def test_mixed_precision_reaches_1e8_against_fp64_operator(ctx):
    s = S.mixed_block(16, seed=1)
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    o.factor_block_jacobi()
    ref, _, _ = o.pcg(100000, 1e-14)
    d = N.DeviceScene(ctx, s)
    d.fit_rotations()
    x0 = s.position.copy()
    st = d.corotational_pass(1e-3, 1e-8, 20000, precision=N.PRECISION_MIXED)
    assert st["converged"] == 1, st
    assert st["true_residual"] <= 1e-8
    err = rel(d.positions() - x0, ref)
    # error against the FP64 oracle solved to its floor; bounded by kappa * 1e-8
    assert err < 1e-5, err


# -- bond stress ----------------------------------------------------------------------------
def test_bond_stress_matches_oracle(ctx):
    s = deformed(S.mixed_block(8, seed=10), seed=11, amp=3e-4)
    o, d, x0, _, st = pass_pair(ctx, s, 1e-3, 1e-12, 5000)
    ro, fo = o.bond_stress()
    g = d.bond_stress()
    rg, fg = g["ratio"].astype(np.float64), g["force"].astype(np.float64)
    assert np.array_equal(ro < 0, rg < 0)
    live = ro >= 0
    # ratios come back as f32
    assert np.all(np.abs(rg[live] - ro[live]) <= 1e-6 * np.maximum(ro[live], 1e-3))
    assert rel(fg, fo) < 1e-6


def test_bond_stress_lists_near_limit_bonds(ctx):
    """A bond driven to exactly its limit appears in the near-limit list."""
    s = S.from_cells([[0, 0, 0], [1, 0, 0]], 3, S.M.table())
    s.fix_voxels([1])  # the fracture loop skips bonds whose owner is kinematic
    o = O.OracleScene(s)
    o.assemble(1e-3)
    frame = o.system_arrays()["frame"][0, 0]
    mk = o.system_arrays()["material_k"][0, 0]
    # stone tension limit 7 MPa: stretch so that k_xx u / AREA = 7e6 exactly
    u = 7e6 * O.VXO_AREA / mk[0, 0]
    s.position[1, 0] += u
    d = N.DeviceScene(ctx, s)
    d.corotational_pass(1e-3, 1e-12, 10)
    d.set_positions(s.position)
    g = d.bond_stress()
    assert abs(g["ratio"][0, 0] - 1.0) < 1e-5
    assert 0 in g["near"].tolist()


# -- compatibility shim (cuda_solver::solve_pcg) ------------------------------------------
def test_shim_analytic_two_node_system():
    from test_oracle_golden import two_node_expected, two_node_rows
    st, dx, it, rel_res = N.solve_pcg_f32(two_node_rows(), 80, 1e-5)
    assert st == N.VX_OK
    assert np.max(np.abs(dx - two_node_expected())) <= 1e-5
    assert rel_res <= 1e-5


@pytest.mark.parametrize("loaded", [True, False])
def test_shim_matches_reference_cuda_sequence_on_wood_cube(loaded):
    s = loaded_wood_cube() if loaded else S.wood_cube()
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    rows = o.pack_rows()
    st_e, dx_e, it_e, res_e = O.cuda_pcg_emulate(rows, 160, 1e-5)
    st_g, dx_g, it_g, res_g = N.solve_pcg_f32(rows, 160, 1e-5)
    assert st_e == st_g == N.VX_OK
    assert it_g == it_e
    assert rel(dx_g, dx_e) < 1e-4


def test_shim_reports_not_converged_like_the_reference():
    s = S.wood_cube()
    o = O.OracleScene(s)
    o.assemble(1e-3)
    rows = o.pack_rows()
    st, dx, it, res = N.solve_pcg_f32(rows, 5, 1e-9)
    assert st == N.VX_NOT_CONVERGED and it == 5 and res > 1e-9
    assert "did not converge" in N.last_error()


def test_shim_rejects_bad_neighbor_index():
    from test_oracle_golden import two_node_rows
    rows = two_node_rows()
    rows["nbr6"] = rows["nbr6"].copy()
    rows["nbr6"][0] = 7
    st, *_ = N.solve_pcg_f32(rows, 10, 1e-5)
    assert st == N.VX_BAD_INPUT


# -- status paths ---------------------------------------------------------------------------
def test_pass_not_converged_status_and_outputs(ctx):
    s = S.wood_cube()
    d = N.DeviceScene(ctx, s)
    st = d.corotational_pass(1e-3, 1e-12, 3)
    assert st["status"] == N.VX_NOT_CONVERGED and st["iterations"] == 3


def test_nonfinite_positions_are_rejected(ctx):
    s = S.wood_cube()
    d = N.DeviceScene(ctx, s)
    bad = s.position.copy()
    bad[5, 1] = np.nan
    with pytest.raises(N.VxError) as e:
        d.set_positions(bad)
    assert e.value.status == N.VX_NONFINITE


def test_empty_scene(ctx):
    s = S.from_cells(np.zeros((0, 3), np.int32), 1, S.M.table())
    d = N.DeviceScene(ctx, s)
    st = d.corotational_pass(1e-3, 1e-8, 10)
    assert st["iterations"] == 0 and st["converged"] == 1
    assert d.fit_rotations() == 0.0


# -- persistent on-chip inner solve ----------------------------------------------------------
@pytest.mark.parametrize("edge", [8, 24])
def test_persistent_inner_solve_matches_streaming_and_oracle(ctx, edge):
    s = S.mixed_block(edge, seed=5)
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    o.factor_block_jacobi()
    ref, _, _ = o.pcg(200000, 1e-14)
    x0 = s.position.copy()
    out = {}
    for kernel in (N.KERNEL_STREAMING, N.KERNEL_PERSISTENT):
        d = N.DeviceScene(ctx, s)
        d.fit_rotations()
        st = d.corotational_pass(1e-3, 1e-8, 50000, precision=N.PRECISION_MIXED, kernel=kernel)
        assert st["converged"] == 1 and st["true_residual"] <= 1e-8, (kernel, st)
        out[kernel] = d.positions() - x0
        d.close()
    for dx in out.values():
        assert rel(dx, ref) < 1e-5
    assert rel(out[N.KERNEL_PERSISTENT], out[N.KERNEL_STREAMING]) < 2e-5


@pytest.mark.parametrize("edge", [48, 64])
def test_persistent_kernels_agree_at_full_grid(ctx, edge):
    """All 148 blocks busy (R = 2 at 48^3, R = 4 at 64^3): both inner kernels
    reach the FP64 target and agree over three passes."""
    s = S.mixed_block(edge, seed=3)
    out = {}
    for kernel in (N.KERNEL_STREAMING, N.KERNEL_PERSISTENT):
        d = N.DeviceScene(ctx, s)
        for _ in range(3):
            d.fit_rotations()
            st = d.corotational_pass(1e-3, 1e-8, 20000, precision=N.PRECISION_MIXED, kernel=kernel)
            assert st["converged"] == 1 and st["true_residual"] <= 1e-8, (kernel, st)
        out[kernel] = d.positions() - s.position
        d.close()
    assert rel(out[N.KERNEL_PERSISTENT], out[N.KERNEL_STREAMING]) < 2e-5


@pytest.mark.parametrize("edge", [24, 64])
def test_persistent_forms_agree(ctx, edge, monkeypatch):
    """The brick plan (Chronopoulos-Gear recurrence, one grid reduction per
    iteration, VXCOROT_PERSISTENT=brick), the contiguous-range plan with the
    classic recurrence (two reductions, VXCOROT_PERSISTENT=range) and with the
    expanded one (one reduction, VXCOROT_PERSISTENT=expanded) all reach the
    FP64 target over three passes, agree to the solve error and take about the
    same number of inner iterations."""
    s = S.mixed_block(edge, seed=3)
    out, iters = {}, {}
    for form in ("brick", "range", "expanded"):
        monkeypatch.setenv("VXCOROT_PERSISTENT", form)
        d = N.DeviceScene(ctx, s)
        it = 0
        for _ in range(3):
            d.fit_rotations()
            st = d.corotational_pass(1e-3, 1e-8, 20000, precision=N.PRECISION_MIXED, kernel=N.KERNEL_PERSISTENT)
            assert st["converged"] == 1 and st["true_residual"] <= 1e-8, (form, st)
            it += st["iterations"]
        assert d.kernel_times(N.PRECISION_MIXED, reps=1)["persistent_form"] == form
        out[form] = d.positions() - s.position
        iters[form] = it
        d.close()
    print(f"{edge}^3 inner iterations over 3 passes: {iters}")
    for form in ("brick", "expanded"):
        assert rel(out[form], out["range"]) < 2e-5, form
        assert abs(iters[form] - iters["range"]) <= 0.05 * iters["range"] + 16, form


def test_wide_plate_takes_the_brick_form(ctx, monkeypatch):
    """A 184 x 184 x 3 plate: its z-neighbour delta (33,856) does not fit the
    range plan's int16 deltas, so the untuned persistent solve takes the brick
    plan, and its result matches the streaming kernels'."""
    monkeypatch.delenv("VXCOROT_PERSISTENT", raising=False)
    cells = S.grid_cells(184, 184, 3)
    s = S.from_cells(cells, 1, S.wood_config_materials(), anisotropy=1.0)
    s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
    free = s.kinematic == 0
    s.loads[free] = np.random.default_rng(4).normal(0.0, 0.05, size=(int(free.sum()), 3))
    out = {}
    for kernel in (N.KERNEL_PERSISTENT, N.KERNEL_STREAMING):
        d = N.DeviceScene(ctx, s)
        d.fit_rotations()
        st = d.corotational_pass(1e-3, 1e-8, 20000, precision=N.PRECISION_MIXED, kernel=kernel)
        assert st["converged"] == 1 and st["true_residual"] <= 1e-8, (kernel, st)
        if kernel == N.KERNEL_PERSISTENT:
            assert d.kernel_times(N.PRECISION_MIXED, reps=1)["persistent_form"] == "brick"
        out[kernel] = d.positions() - s.position
        d.close()
    assert rel(out[N.KERNEL_PERSISTENT], out[N.KERNEL_STREAMING]) < 2e-5


def test_persistent_solve_on_wood_cube_meets_fp64_target(ctx):
    s = loaded_wood_cube()
    d = N.DeviceScene(ctx, s)
    d.fit_rotations()
    st = d.corotational_pass(1e-3, 1e-10, 20000, precision=N.PRECISION_MIXED, kernel=N.KERNEL_PERSISTENT)
    assert st["converged"] == 1 and st["true_residual"] <= 1e-10, st


@pytest.mark.parametrize("form", ["brick", "range", "expanded"])
def test_persistent_barrier_wait_runs_out_and_reports_timeout(form):
    """A wait bounded at one poll runs out (no block is missing, the bound is
    simply too small): in the brick form the neighbour-flag wait or the grid
    reduction, in the range forms a grid reduction. The kernel records
    VX_TIMEOUT and returns, and the context stays usable."""
    import subprocess
    import sys
    import textwrap
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = textwrap.dedent(f"""
        import sys
        sys.path[:0] = [{str(root / 'voxel-sim_b200')!r}]
        from vxsim import native as N, scenes as S
        ctx = N.Context(0)
        d = N.DeviceScene(ctx, S.mixed_block(24, seed=5))
        d.fit_rotations()
        try:
            d.corotational_pass(1e-3, 1e-8, 5000, precision=N.PRECISION_MIXED, kernel=N.KERNEL_PERSISTENT)
            print("NO_TIMEOUT")
        except N.VxError as e:
            print("STATUS", e.status)
        st = d.corotational_pass(1e-3, 1e-8, 5000, precision=N.PRECISION_MIXED, kernel=N.KERNEL_STREAMING)
        print("AFTER", st["converged"])
    """)
    env = dict(__import__("os").environ, VXCOROT_BARRIER_SPINS="1", VXCOROT_PERSISTENT=form)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert f"STATUS {N.VX_TIMEOUT}" in out.stdout, out.stdout + out.stderr
    assert "AFTER 1" in out.stdout
