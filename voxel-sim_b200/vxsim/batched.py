"""Batched form: many independent scenes solved together in one pool.

The batched workload is 512 scenes, each a random union of 1-4 axis-aligned
boxes in a cube whose edge is log-uniform over 8-48 REVs, with a random
material and grain, one face clamped and the opposite face displaced 0.05 mm
(scenes.box_union_scene). A batched solve is one corotational pass of every
scene (rotation fit, assembly, FP32 inner PCG in FP64 refinement to 1e-8)
through vx_pool_fit_rotations / vx_pool_pass. The same scenes solved one at
a time in the plain FP64 form (vx_corotational_pass, VX_PRECISION_FP64) are
the comparison.
"""
from __future__ import annotations

import numpy as np

from . import native as N
from . import scenes as S

TILE = 256


def batched_scenes(count: int = 512, seed: int = 2024, edge_lo: int = 8, edge_hi: int = 48):
    rng = np.random.default_rng(seed)
    return [S.box_union_scene(rng, edge_lo, edge_hi) for _ in range(count)]


def pool_capacity(scenes) -> int:
    return sum((s.n + TILE - 1) // TILE * TILE for s in scenes)


class BatchedSolve:
    """Every scene resident in one pool; solve() runs one pass of all of them
    from the state saved at construction."""

    def __init__(self, ctx: N.Context, scenes, h: float = 1e-3, tolerance: float = 1e-8,
                 max_iterations: int = 20000, kernel: int = N.KERNEL_AUTO):
        self.scenes = scenes
        self.kernel = kernel
        self.pool = N.DevicePool(ctx, pool_capacity(scenes), len(scenes))
        self.slots = [self.pool.add(s) for s in scenes]
        self.h, self.tolerance, self.max_iterations = h, tolerance, max_iterations
        self.pool.save_state()

    @property
    def stream_ptr(self) -> int:
        return self.pool.stream_ptr

    def solve(self):
        self.pool.restore_state()
        self.pool.fit_rotations()
        status, stats = self.pool.corotational_pass(self.h, self.tolerance, self.max_iterations, kernel=self.kernel)
        return status, [stats[k] for k in self.slots]

    def close(self):
        self.pool.close()


class SingleSceneSolves:
    """The same scenes as separate resident scenes, each solved alone in the
    plain FP64 form."""

    def __init__(self, ctx: N.Context, scenes, h: float = 1e-3, tolerance: float = 1e-8,
                 max_iterations: int = 20000):
        self.h, self.tolerance, self.max_iterations = h, tolerance, max_iterations
        self.devs = []
        for s in scenes:
            d = N.DeviceScene(ctx, s)
            d.save_state()
            self.devs.append(d)

    def solve(self, k: int):
        d = self.devs[k]
        d.restore_state()
        d.fit_rotations()
        return d.corotational_pass(self.h, self.tolerance, self.max_iterations, precision=N.PRECISION_FP64)

    def close(self):
        for d in self.devs:
            d.close()
