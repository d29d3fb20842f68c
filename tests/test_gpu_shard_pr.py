"""Sample sharding of one PR-MPPI controller across processes (dr_prmppi_set_shard /
dr_prmppi_shard_*): two processes, each with half of the samples under every hypothesis,
exchanging their minima and weighted sums (taken with their own minima) by one all-gather,
against one process stepping the whole controller.

The processes share the one GPU of the test box; their kernels never wait on one
another (the exchange happens on the host between the phases, over gloo), so this is
the multi-process path exactly as it runs with one GPU per process, minus NCCL."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import drb

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
STEPS = 3


def _scenario():
    sys.path.insert(0, str(ROOT / "tests"))
    from test_gpu_prmppi import small_pr

    return small_pr(8, K=2048, T=40, noise=True)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _record(ctl):
    i = ctl.info
    return (bool(i.use_nom_plan), bool(i.reset_nom), tuple(float(x) for x in i.min_costs), tuple(float(x) for x in i.nu),
            tuple(float(x) for x in i.cand_cost))


def _worker(rank: int, world: int, port: int, q) -> None:
    try:
        sys.path.insert(0, str(ROOT / "tests"))
        sys.path.insert(0, str(ROOT))
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import torch.distributed as dist

        dist.init_process_group("gloo", rank=rank, world_size=world)
        from conftest import drb as pkg

        sc = _scenario()
        ctl = pkg.controllers.ShardedPRMPPIController(sc.env, sc.prmppi, sc.seed, rank, world)
        ctl.engine = object()
        acts, noms, recs = [], [], []
        for _ in range(STEPS):
            acts.append(ctl.getControl(sc.state))
            noms.append(np.concatenate(ctl.nominals()))
            recs.append(_record(ctl))
        q.put((rank, acts, noms, recs, None))
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, None, None, None, repr(e)))


def test_two_pr_shards_equal_one_controller(gpu):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, acts, noms, recs, err = q.get(timeout=300)
        assert err is None, err
        res[rank] = (acts, noms, recs)
    for p in procs:
        p.join(timeout=60)
    sc = _scenario()
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed)
    ctl.engine = object()
    with pytest.raises(drb.abi.DrError):
        bad = drb.controllers.ShardedPRMPPIController(sc.env, sc.prmppi, sc.seed, 0, 2)
        bad.engine = object()
        drb.controllers.PRMPPIController.getControl(bad, sc.state)  # the single-process step is refused
    for k in range(STEPS):
        a = ctl.getControl(sc.state)
        nom = np.concatenate(ctl.nominals())
        rec = _record(ctl)
        for r in (0, 1):
            acts, noms, recs = res[r]
            # the shards agree with each other exactly (same gathered partials, merged alike)
            assert np.array_equal(acts[k], res[0][0][k]) and np.array_equal(noms[k], res[0][1][k]) and recs[k] == res[0][2][k]
            # and with the single process to FP32 rounding (the rescaled sums round differently)
            np.testing.assert_allclose(acts[k], a, rtol=1e-4, atol=1e-5)
            np.testing.assert_allclose(noms[k], nom, rtol=1e-4, atol=1e-5)
            assert recs[k][0] == rec[0] and recs[k][1] == rec[1]
            assert recs[k][2] == rec[2]  # minima are exact
            np.testing.assert_allclose(recs[k][3], rec[3], rtol=1e-4)
            np.testing.assert_allclose(recs[k][4], rec[4], rtol=1e-4, atol=1e-3)
    print("shard actions", [res[0][0][k] for k in range(STEPS)], "decisions", [res[0][2][k][:2] for k in range(STEPS)])
