"""The replica form of bench.py --gpus N on CPU: two gloo ranks combine their
timings and work as the NCCL ranks do (maximum device time, summed work)."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [120.0, 150.0][rank]
    work = [1.0e9, 3.0e9][rank]
    got = bench.combine_ranks(ms, work, 5.0, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_two_gloo_ranks_combine_like_the_nccl_run():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert results[r] == (150.0, 4.0e9, 10.0)


def test_single_rank_passes_figures_through():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.combine_ranks(10.0, 2.0, 3.0) == (10.0, 2.0, 3.0)
