"""Served form: a Poisson stream of scene-step requests through vx_server.

Each request is a wood block built as in the batched workload (a union of
1-4 axis-aligned boxes spanning the cube; size log-uniform over 1k-2M DOF,
grain random) whose bottom layer is clamped and whose top face is pressed by
a blade (a 2 x 20 REV footprint of a 2 x 20 x 40 iron blade, centred on the
top face, with a one-REV bevel: the two rows of its edge) driven into the
block at 1 m/s. The blade itself is not simulated: contact with it is the
prescribed displacement of the wood REVs under its edge, which are targeted
and advance at the blade speed every step (tools and contact projection are
outside the elastic path). Each request runs 100 fixed steps of 1 ms with
its state resident on the device; admission is capped by the pool, sized at
80% of the device memory.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import native as N
from . import scenes as S


def served_scene(rng, dof_lo: float = 1e3, dof_hi: float = 2e6) -> tuple:
    """(scene, moving mask) for one request. The boxes are drawn as fractions of
    the cube edge, then the edge is chosen so the union holds about the drawn
    REV count (DOF / 3)."""
    revs = math.exp(rng.uniform(math.log(dof_lo / 3.0), math.log(dof_hi / 3.0)))
    boxes = []
    for _ in range(int(rng.integers(1, 5))):
        a, b = rng.random(3), rng.random(3)
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        lo[2], hi[2] = 0.0, 1.0  # every box spans the height, so the clamped bottom holds it
        boxes.append((lo, hi))

    def raster(edge):
        occ = np.zeros((edge, edge, edge), bool)
        for lo, hi in boxes:
            i0 = np.floor(lo * edge).astype(int)
            i1 = np.maximum(np.ceil(hi * edge).astype(int), i0 + 1)
            occ[i0[0]:i1[0], i0[1]:i1[1], i0[2]:i1[2]] = True
        return occ

    edge = max(3, int(round(revs ** (1.0 / 3.0))))
    fill = raster(edge).mean()
    edge = max(3, int(round((revs / fill) ** (1.0 / 3.0))))
    x, y, z = np.nonzero(raster(edge))
    cells = np.stack([x, y, z], axis=1).astype(np.int32)
    cells = cells[np.lexsort((cells[:, 0], cells[:, 1], cells[:, 2]))]
    table = S.wood_config_materials()
    g = S.random_unit_vectors(rng, 1)[0]
    n = len(cells)
    s = S.from_cells(cells, 1, table, fiber=np.tile(g, (n, 1)), anisotropy=1.0)
    s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
    # blade edge: 2 rows (the bevel) x 20 REVs along y, centred over the top face's cells
    top = cells[:, 2] == edge - 1
    cx, cy = int(np.round(cells[top, 0].mean())), int(np.round(cells[top, 1].mean()))
    under = top & (cells[:, 0] >= cx) & (cells[:, 0] <= cx + 1) & (cells[:, 1] >= cy - 10) & (cells[:, 1] < cy + 10)
    s.target_mask[under] = 7
    s.target[under] = s.position[under]
    s.meta.update(workload="served", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, -9.81))
    return s, under


def run_served(ctx: N.Context, rate: float = 200.0, duration: float = 5.0, steps: int = 100,
               max_slots: int = 256, templates: int = 16, seed: int = 77, drain: float = 60.0,
               blade_speed: float = 1.0, hbm_fraction: float = 0.8, tolerance: float = 1e-8) -> dict:
    rng = np.random.default_rng(seed)
    pool = [served_scene(rng) for _ in range(templates)]
    params = N.step_params(1e-3, substeps=1, corotation_iterations=2, corotation_tolerance=1e-5,
                           gravity=(0.0, 0.0, -9.81), tolerance=tolerance, max_iterations=20000,
                           precision=N.PRECISION_MIXED)
    srv = N.Server(ctx, params, max_slots=max_slots, hbm_fraction=hbm_fraction)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * duration * 2) + 16))
    arrivals = arrivals[arrivals < duration]
    picks = rng.integers(0, templates, size=len(arrivals))
    tickets, sizes = [], []
    t0 = time.perf_counter()
    for t, k in zip(arrivals, picks):
        now = time.perf_counter() - t0
        if t > now:
            time.sleep(t - now)
        scene, moving = pool[k]
        tickets.append(srv.submit(scene, steps, target_velocity=(0.0, 0.0, -blade_speed), moving=moving))
        sizes.append(scene.n)
    submit_s = time.perf_counter() - t0
    results = []
    deadline = time.perf_counter() + drain
    for tk in tickets:
        left = deadline - time.perf_counter()
        r = srv.wait(tk, max(0.0, left)) if left > 0 else None
        if r is not None:
            results.append(r[0])
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    done = [r for r in results if r["status"] in (N.VX_OK, N.VX_NOT_CONVERGED)]
    return {
        "requests": len(tickets), "completed": len(done), "arrival_rate": rate, "arrival_window_s": duration,
        "submit_s": submit_s, "wall_s": wall, "steps_per_request": steps,
        "dof_range": [3 * min(sizes) if sizes else 0, 3 * max(sizes) if sizes else 0],
        "templates": templates, "stats": st,
        "not_converged": sum(1 for r in done if r["status"] == N.VX_NOT_CONVERGED),
        "worst_residual": max((r["worst_residual"] for r in done), default=None),
        "mean_queued_s": float(np.mean([r["queued_s"] for r in done])) if done else None,
    }
