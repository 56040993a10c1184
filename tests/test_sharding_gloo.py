"""Scene sharding over ranks (vxsim.sharding) on CPU: the assignment, and two
gloo ranks solving one batch with the results gathered on rank 0.

The per-rank solve is replaced, in this test only, by a CPU stand-in that
returns a digest of each scene; on a GPU job it is sharding.pool_pass (the
rank's scenes in one pool on its device). The test checks that every scene is
solved exactly once, by the rank the assignment names, and that the gathered
results equal a single-rank run."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path[:0] = [str(ROOT / "voxel-sim_b200")]

from vxsim import scenes as S  # noqa: E402
from vxsim import sharding as H  # noqa: E402


def batch():
    rng = np.random.default_rng(11)
    return [S.box_union_scene(rng, 4, 12) for _ in range(13)]


def stand_in(tag):
    def solve(local):
        return [{"n": s.n, "digest": float(np.round(s.position.sum(), 9)), "by": tag} for s in local]
    return solve


def test_assignment_covers_every_scene_once_and_balances_revs():
    sizes = [s.n for s in batch()]
    for world in (1, 2, 3, 5):
        parts = H.assign(sizes, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in p) for p in parts]
        # longest-processing-time: no rank exceeds the mean by more than the largest scene
        assert max(loads) - min(loads) <= max(sizes)
        assert H.assign(sizes, world) == parts  # deterministic


def test_single_process_solves_all_in_order():
    scenes = batch()
    out = H.solve_sharded(scenes, stand_in("solo"))
    assert [r["n"] for r in out] == [s.n for s in scenes]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path[:0] = [str(ROOT / "voxel-sim_b200")]
    from vxsim import sharding as Hs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    out = Hs.solve_sharded(batch(), stand_in(rank), dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def test_two_gloo_ranks_shard_and_gather_like_one_rank():
    scenes = batch()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    gathered = got[0]
    parts = H.assign([s.n for s in scenes], 2)
    for r, part in enumerate(parts):
        assert part and all(gathered[k]["by"] == r for k in part)
    solo = H.solve_sharded(scenes, stand_in("solo"))
    strip = lambda rs: [{k: v for k, v in r.items() if k != "by"} for r in rs]
    assert strip(gathered) == strip(solo)
