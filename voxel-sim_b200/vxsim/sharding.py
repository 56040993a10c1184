"""One batch of independent scenes spread over the ranks of a job.

Scenes share nothing, so a batch shards by whole scenes: every rank (one
process per GPU) takes a share, solves it in a pool on its own device with the
scenes' state resident there, and the results are gathered on rank 0's host.
There is no collective on the data path; the only communication is the final
host gather of each rank's results (torch.distributed object gather, gloo or
NCCL process group).

The assignment is longest-processing-time first: scenes in decreasing REV
count go to the rank with the fewest REVs so far (ties to the lower rank, then
the lower scene index), so the ranks' pools hold about equal REV counts and
every rank computes the same assignment without communicating.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def assign(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Scene indices per rank (each list in increasing index order)."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(v) for v in out]


def solve_sharded(scenes: Sequence, solve_local: Callable[[list], list], dist=None):
    """Solve `scenes` over the ranks of `dist` (None: this process alone).

    solve_local(list_of_scenes) -> list of per-scene results, run by every rank
    on its share. Returns the results in scene order on rank 0 and None on the
    other ranks. Every rank takes the same steps in the same order."""
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    mine = assign([s.n for s in scenes], world)[rank]
    results = solve_local([scenes[k] for k in mine]) if mine else []
    if len(results) != len(mine):
        raise RuntimeError(f"rank {rank}: {len(results)} results for {len(mine)} scenes")
    pairs = list(zip(mine, results))
    if dist is None:
        gathered = [pairs]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(pairs, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(scenes)
    for part in gathered:
        for k, res in part:
            if out[k] is not None:
                raise RuntimeError(f"scene {k} solved twice")
            out[k] = res
    missing = [k for k, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"scenes not solved: {missing[:8]}")
    return out


def pool_pass(ctx, h: float = 1e-3, tolerance: float = 1e-8, max_iterations: int = 20000):
    """solve_local for solve_sharded: the rank's scenes resident in one pool on
    `ctx`'s device, one corotational pass each (rotation fit, assembly, FP32
    inner PCG in FP64 refinement to `tolerance`); per scene its displacement
    and pass statistics."""
    from . import native as N
    from .batched import BatchedSolve

    def solve(local_scenes: list) -> list:
        bs = BatchedSolve(ctx, local_scenes, h=h, tolerance=tolerance, max_iterations=max_iterations)
        try:
            status, stats = bs.solve()
            if status not in (N.VX_OK, N.VX_NOT_CONVERGED):
                raise N.VxError(status, N.last_error())
            return [{"displacement": bs.pool.positions(slot) - s.position, "stats": st}
                    for s, slot, st in zip(local_scenes, bs.slots, stats)]
        finally:
            bs.close()

    return solve
