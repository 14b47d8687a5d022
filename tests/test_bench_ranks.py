"""The multi-rank plumbing of bench.py (replicas: one independent batch per
rank, no data-path collective) on CPU with gloo, world size 2: the timing
is the max over ranks, every rank takes the same collective steps, the
replicas draw different problems, and only rank 0 reports."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    import argparse
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from cup2d_b200.problems import batch_problems
        bench._barrier(world)
        worst = bench._max_over_ranks(1.5 + rank, world)
        meshes = batch_problems(4, seed=3 + 1000 * rank, lo=50, hi=200)
        args = argparse.Namespace(impl="reference", workload="batch")
        ref = bench.run_reference(args, world, rank) if rank != 0 else "skipped"
        q.put((rank, worst, [m.nblocks for m in meshes], ref))
        bench._barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, worst, sizes, ref = q.get(timeout=120)
        out[rank] = (worst, sizes, ref)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 2.5          # max over ranks, seen by all
    assert out[0][1] != out[1][1]                  # independent replicas
    assert out[1][2] is None                       # the reference arm: rank 0 alone
