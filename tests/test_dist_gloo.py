"""The N > 1 path of bench.py on CPU ranks (gloo, world size 2): each rank builds its own
independent 4-agent race (replicas, no data-path collective), the timing is the max over
ranks, and every rank takes the same collective steps."""
from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        scs = bench.workload(rank)
        seeds = [s.seed for s in scs]
        t = bench._max_over_ranks(1.0 + rank, world, device="cpu")
        bench._barrier(world)
        out.put((rank, seeds, t, [float(s.env.track_length) for s in scs]))
    finally:
        dist.destroy_process_group()


def test_replicas_over_two_cpu_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, seeds0, t0, len0), (r1, seeds1, t1, len1) = res
    assert t0 == t1 == 2.0  # max over ranks
    assert set(seeds0).isdisjoint(seeds1)  # each rank drives its own race
    assert len(set(seeds0)) == 4
    assert len0 != len1  # different seeded tracks per rank
