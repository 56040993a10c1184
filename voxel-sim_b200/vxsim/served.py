"""Served form: a Poisson stream of scene-step requests through vx_server.

Each request is a wood block built as in the batched workload (a union of
1-4 axis-aligned boxes spanning the cube; size log-uniform over 1k-2M DOF,
grain random) whose bottom layer is clamped, with a 2 x 20 x 40 iron blade
standing on the centre of its top face. The blade is kinematic REVs whose
targets advance at 1 m/s into the block; its lowest row is one REV thick
(the bevel). The blade pushes the wood through the contact stage of the step
(collision::project and the contact velocities), and the wood's bonds go
through the fracture stage. Each request runs 100 fixed steps of 1 ms with
its state resident on the device; admission is capped by the pools, sized at
80% of the device memory together with the contact buffers. The server runs
three lanes by scene size (up to 16,384 REVs, up to 131,072, larger), each
with its own pool, stream and thread.

`blade="targets"` builds the earlier stand-in instead: no blade REVs, the
wood REVs under the blade's edge are targeted and driven at the blade speed.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import native as N
from . import scenes as S


def served_scene(rng, dof_lo: float = 1e3, dof_hi: float = 2e6, blade: str = "contact", dof=None) -> tuple:
    """(scene, moving mask) for one request. The boxes are drawn as fractions of
    the cube edge, then the edge is chosen so the union holds about the drawn
    REV count (DOF / 3) of wood: `dof` when given, else log-uniform over
    [dof_lo, dof_hi]."""
    revs = (dof if dof is not None else math.exp(rng.uniform(math.log(dof_lo), math.log(dof_hi)))) / 3.0
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
    top = cells[:, 2] == edge - 1
    cx, cy = int(np.round(cells[top, 0].mean())), int(np.round(cells[top, 1].mean()))
    n_wood = len(cells)
    if blade == "targets":
        s = S.from_cells(cells, 1, table, fiber=np.tile(g, (n_wood, 1)), anisotropy=1.0)
        s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
        # the wood under the blade's edge: 2 rows x 20 REVs along y
        under = top & (cells[:, 0] >= cx) & (cells[:, 0] <= cx + 1) & (cells[:, 1] >= cy - 10) & (cells[:, 1] < cy + 10)
        s.target_mask[under] = 7
        s.target[under] = s.position[under]
        s.meta.update(workload="served", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, -9.81), wood_revs=n_wood)
        return s, under
    # the blade: 2 (x) x 20 (y) x 40 (z) iron REVs on the top face, lowest row 1 REV thick
    bx, by, bz = np.meshgrid(np.arange(cx, cx + 2), np.arange(cy - 10, cy + 10), np.arange(edge, edge + 40),
                             indexing="ij")
    bcells = np.stack([bx.ravel(), by.ravel(), bz.ravel()], axis=1).astype(np.int32)
    bcells = bcells[(bcells[:, 2] > edge) | (bcells[:, 0] == cx)]
    bcells = bcells[np.lexsort((bcells[:, 0], bcells[:, 1], bcells[:, 2]))]
    all_cells = np.concatenate([cells, bcells])
    n = len(all_cells)
    is_blade = np.arange(n) >= n_wood
    mats = np.where(is_blade, 2, 1).astype(np.uint32)
    fib = np.tile(np.array([0, 0, 1], np.float32), (n, 1))
    fib[:n_wood] = g
    s = S.from_cells(all_cells, mats, table, kinematic=is_blade.astype(np.uint8), fiber=fib,
                     anisotropy=np.where(is_blade, 0.0, 1.0).astype(np.float32))
    s.fix_voxels(np.nonzero(all_cells[:n_wood, 2] == 0)[0])
    s.target_mask[is_blade] = 7
    s.target[is_blade] = s.position[is_blade]
    s.meta.update(workload="served", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, -9.81), wood_revs=n_wood)
    return s, is_blade


def run_served(ctx: N.Context, rate: float = 200.0, duration: float = 5.0, steps: int = 100,
               max_slots: int = 256, templates: int = 16, seed: int = 77, drain: float = 60.0,
               blade_speed: float = 1.0, hbm_fraction: float = 0.8, tolerance: float = 1e-8,
               blade: str = "contact", lanes: int = 3) -> dict:
    rng = np.random.default_rng(seed)
    # the templates' sizes are a log-spaced grid over 1k-2M DOF (the stratified
    # form of log-uniform: the extremes of the range are always present)
    grid = np.exp(np.linspace(math.log(1e3), math.log(2e6), templates))
    pool = [served_scene(rng, blade=blade, dof=float(d)) for d in grid]
    real = blade == "contact"
    params = N.step_params(1e-3, substeps=1, corotation_iterations=2, corotation_tolerance=1e-5,
                           gravity=(0.0, 0.0, -9.81), tolerance=tolerance, max_iterations=20000,
                           precision=N.PRECISION_MIXED, fracture=real, contact=real)
    srv = N.Server(ctx, params, max_slots=max_slots, hbm_fraction=hbm_fraction, lanes=lanes)
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
        sizes.append(scene.meta["wood_revs"])
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
    latency = [r["queued_s"] + r["run_s"] for r in done]
    return {
        "request_latency_s": {"p50": float(np.percentile(latency, 50)) if latency else None,
                              "p99": float(np.percentile(latency, 99)) if latency else None,
                              "max": float(max(latency)) if latency else None},
        "request_solves": int(sum(r["passes"] for r in done)),
        "requests": len(tickets), "completed": len(done), "arrival_rate": rate, "arrival_window_s": duration,
        "blade": blade, "lanes": lanes,
        "submit_s": submit_s, "wall_s": wall, "steps_per_request": steps,
        "dof_range": [3 * min(sizes) if sizes else 0, 3 * max(sizes) if sizes else 0],
        "templates": templates, "stats": st,
        "not_converged": sum(1 for r in done if r["status"] == N.VX_NOT_CONVERGED),
        "worst_residual": max((r["worst_residual"] for r in done), default=None),
        "mean_queued_s": float(np.mean([r["queued_s"] for r in done])) if done else None,
        "template_scenes": [(s, m) for s, m in pool], "template_picks": picks.tolist(),
    }


def single_scene_step_rate(ctx: N.Context, templates, precision: int, steps: int = 4, tolerance: float = 1e-8,
                           blade_speed: float = 1.0, blade: str = "contact") -> dict:
    """The single-scene form on the served requests' own steps: each template
    (scene, moving mask) resident alone, stepped `steps` times as a request
    is (prediction under gravity, two corotational passes, contact and
    fracture with the blade advancing 1 mm per step), timed with CUDA events on
    the scene's stream around each step. Per template: seconds and solves."""
    import torch
    real = blade == "contact"
    params = N.step_params(1e-3, substeps=1, corotation_iterations=2, corotation_tolerance=1e-5,
                           gravity=(0.0, 0.0, -9.81), tolerance=tolerance, max_iterations=200000,
                           precision=precision, fracture=real, contact=real)
    out = []
    for s, moving in templates:
        d = N.DeviceScene(ctx, s)
        mask = np.ascontiguousarray(s.target_mask, np.uint8)
        target = np.array(s.target, np.float64)
        ext = torch.cuda.ExternalStream(d.stream_ptr)
        secs, solves, worst = 0.0, 0, 0.0
        for _ in range(steps):
            target[np.asarray(moving, bool), 2] -= blade_speed * 1e-3
            d.set_targets(mask, target)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            st = d.step(params)
            e1.record(ext)
            e1.synchronize()
            secs += e0.elapsed_time(e1) / 1000.0
            solves += st["passes"]
            worst = max(worst, st["residual"])
        d.close()
        out.append({"n": s.n, "seconds": secs, "solves": solves, "worst_residual": worst})
    return out
