"""Sample sharding of one controller across processes (dr_mppi_set_shard /
dr_mppi_shard_*): two processes, each with half of the samples and half of the
verification samples, exchanging their partial minima, weighted sums (taken with their own
minima) and previous-plan failure histograms by one all-gather and the new plan's
histograms by one all-reduce, against one process stepping the whole controller.

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
import helpers as H

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
STEPS = 3


def _scenario(spl: bool):
    sc = H.small_mppi(spl, K=1024, T=40, n_verif=2048, seed=9, noise=True)
    sc.mppi.max_verif_eps = 0.01  # lets new plans certify with 2048 samples
    return sc


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, spl: bool, q) -> None:
    try:
        sys.path.insert(0, str(ROOT / "tests"))
        sys.path.insert(0, str(ROOT))
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import torch.distributed as dist

        dist.init_process_group("gloo", rank=rank, world_size=world)
        from conftest import drb as pkg

        sc = _scenario(spl)
        ctl = pkg.controllers.ShardedMPPIController(sc.env, sc.mppi, sc.seed, rank, world)
        ctl.engine = object()
        acts, noms, fcs, infos = [], [], [], []
        for _ in range(STEPS):
            acts.append(ctl.getControl(sc.state))
            noms.append(ctl.h_nominal)
            fcs.append(ctl.failCount.copy())
            infos.append((ctl.info.use_new_plan, ctl.info.fail_count_total, ctl.info.nu, ctl.info.min_cost))
        q.put((rank, acts, noms, fcs, infos, None))
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, None, None, None, None, repr(e)))


@pytest.mark.parametrize("spl", [True, False])
def test_two_shards_equal_one_controller(gpu, spl):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, spl, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, acts, noms, fcs, infos, err = q.get(timeout=300)
        assert err is None, err
        res[rank] = (acts, noms, fcs, infos)
    for p in procs:
        p.join(timeout=60)
    # the whole controller in this process
    sc = _scenario(spl)
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed)
    ctl.engine = object()
    for k in range(STEPS):
        a = ctl.getControl(sc.state)
        nom = ctl.h_nominal
        for r in (0, 1):
            acts, noms, fcs, infos = res[r]
            # the two shards agree with each other exactly (same gathered partials, merged alike)
            assert np.array_equal(acts[k], res[0][0][k]) and np.array_equal(noms[k], res[0][1][k])
            # and with the single process to FP32 rounding (the rescaled sums round differently)
            np.testing.assert_allclose(acts[k], a, rtol=1e-4, atol=1e-5)
            np.testing.assert_allclose(noms[k], nom, rtol=1e-4, atol=1e-5)
            assert infos[k][0] == ctl.info.use_new_plan
            assert abs(int(infos[k][1]) - int(ctl.info.fail_count_total)) <= 2
            assert abs(int(fcs[k].sum()) - int(ctl.failCount.sum())) <= 2
            assert infos[k][3] == ctl.info.min_cost  # minima are exact
            np.testing.assert_allclose(infos[k][2], ctl.info.nu, rtol=1e-4)
    print("shard actions", [res[0][0][k] for k in range(STEPS)])
