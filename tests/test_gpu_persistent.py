"""Persistent launches fed by a device work queue (dr_mppi_batch_set_persistent) and the
launch-shape autotuner (dr_mppi_batch_autotune) on a batch of uneven races: controllers
of different tracks, sample counts, horizons and verification sizes. Every launch shape
must give the same actions, plans and failure histograms, bit for bit, as the
one-CTA-per-tile grid: tiles are independent, and the histograms are integer sums."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import drb
import helpers as H

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios

# (track seed, K, T, n_verif, gradient steps)
SIZES = [(0, 256, 32, 700, 0), (1, 1500, 48, 2048, 3), (2, 640, 64, 1300, 0), (3, 4096, 24, 512, 2), (4, 96, 40, 3000, 0)]
# constant warm starts of the small strategic race that crash within the verification
# horizon, so that the histograms hold failures and the plan choice goes both ways
CRASH = {0: [0.0, 3.0], 2: [3.0, 0.0], 3: [0.0, 0.0]}


def _controllers(spl: bool, grad: bool):
    scs, ctls = [], []
    for i, (seed, k, t, v, g) in enumerate(SIZES):
        if i in CRASH:
            s = H.small_mppi(spl, K=k, T=t, n_verif=v, seed=11 + i, noise=True)
            s.mppi.max_verif_eps = 0.01
            nom = np.tile(np.array(CRASH[i], np.float32), (s.n_theta + 1, s.mppi.n_timesteps, 1))
        else:
            s = S.circle_race(agent=i, seed=seed, K=k, T=t, n_verif=v, use_splines=spl)
            nom = None
        c = drb.controllers.MPPIController(s.env, s.mppi, s.seed, nominal=nom)
        if grad and g:
            c.set_grad_refine(g, 0.05, 0)
        scs.append(s)
        ctls.append(c)
    return scs, ctls


def _run(spl: bool, grad: bool, shape, steps: int = 3, tune: bool = False):
    scs, ctls = _controllers(spl, grad)
    batch = drb.controllers.MPPIBatch(ctls)
    beliefs = np.stack([s.belief() for s in scs])
    out, report = [], None
    for k in range(steps):
        if k == 1:
            if tune:
                report = batch.autotune(3)
            elif shape is not None:
                batch.set_persistent(*shape)
        a = batch.step([s.state for s in scs], beliefs)
        for c in ctls:
            c._pull()  # the batch step leaves the histograms on the controllers' handles
        out.append((a.copy(), [c.h_nominal.copy() for c in ctls], [np.concatenate([c.failCountNew, c.failCountOld]) for c in ctls],
                    [(c.info.use_new_plan, c.info.nu, c.info.min_cost) for c in ctls]))
    return out, report


def _same(x, y):
    for (a1, n1, f1, i1), (a2, n2, f2, i2) in zip(x, y):
        assert np.array_equal(a1, a2)
        for u, v in zip(n1, n2):
            assert np.array_equal(u, v)
        for u, v in zip(f1, f2):
            assert np.array_equal(u, v)
        assert i1 == i2


@pytest.mark.parametrize("spl", [True, False])
@pytest.mark.parametrize("shape", [(-1, -1, 0), (1, 1, 1), (2, 0, 0), (0, 1, 1), (0, 0, 1)])
def test_persistent_equals_static_grid(gpu, spl, shape):
    ref, _ = _run(spl, False, None)
    got, _ = _run(spl, False, shape)
    _same(ref, got)
    # the histograms did count failures (the comparison is not vacuous)
    assert any(int(f.sum()) > 0 for step in ref for f in step[2])


@pytest.mark.parametrize("side,pdl", [(0, True), (1, False), (-1, True)])
def test_side_verification_shape(gpu, side, pdl):
    """The previous plan's verification beside the rollout as one CTA per tile or as a
    persistent grid: the same results as the default."""
    ref, _ = _run(True, False, None)
    scs, ctls = _controllers(True, False)
    batch = drb.controllers.MPPIBatch(ctls)
    batch.set_side_verify(side)
    batch.set_pdl(pdl)
    beliefs = np.stack([s.belief() for s in scs])
    got = []
    for _ in range(3):
        a = batch.step([s.state for s in scs], beliefs)
        for c in ctls:
            c._pull()
        got.append((a.copy(), [c.h_nominal.copy() for c in ctls], [np.concatenate([c.failCountNew, c.failCountOld]) for c in ctls],
                    [(c.info.use_new_plan, c.info.nu, c.info.min_cost) for c in ctls]))
    _same(ref, got)


def test_autotune_keeps_results_and_reports(gpu):
    ref, _ = _run(True, True, None)
    got, rep = _run(True, True, None, tune=True)
    _same(ref, got)
    print("autotune:", rep)
    assert (0, 0) in rep["rollout"] and (0, 1) in rep["rollout"] and len(rep["rollout"]) >= 4
    assert 0 in rep["verify"] and len(rep["verify"]) >= 2
    assert len(rep["grad"]) >= 2
    assert (rep["rollout_ctas_per_sm"], rep["rollout_lockstep"]) in rep["rollout"]
    assert rep["verify_ctas_per_sm"] in rep["verify"]
    assert rep["grad_ckpt"] in rep["grad"]
    assert all(v > 0 for d in ("rollout", "verify", "grad") for v in rep[d].values())


def test_persistent_device_resident_loop(gpu):
    """The persistent shapes inside the graph-replayed device-resident closed loop."""
    import torch

    def loop(shape):
        scs, ctls = _controllers(True, False)
        batch = drb.controllers.MPPIBatch(ctls)
        n = len(scs)
        states = torch.from_numpy(np.frombuffer(bytes((abi.dr_sim_state * n)(*[s.state for s in scs])), np.uint8).copy()).cuda()
        bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
        bel[:, :2] = np.stack([s.belief() for s in scs])
        beliefs = torch.from_numpy(bel).cuda()
        actions = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
        infos = torch.zeros(n * ctypes.sizeof(abi.dr_mppi_info), dtype=torch.uint8, device="cuda")
        theta = torch.zeros(n, dtype=torch.int32, device="cuda")
        terms = torch.zeros(n, dtype=torch.int32, device="cuda")
        if shape is not None:
            batch.set_persistent(*shape)
        torch.cuda.synchronize()
        acts = []
        for _ in range(4):
            batch.step_device(states.data_ptr(), beliefs.data_ptr(), actions.data_ptr(), infos.data_ptr())
            batch.env_step_device(theta.data_ptr(), actions.data_ptr(), states.data_ptr(), beliefs.data_ptr(), True, 5, terms.data_ptr())
            torch.cuda.synchronize()
            acts.append(actions.cpu().numpy().copy())
        return np.stack(acts)

    assert np.array_equal(loop(None), loop((-1, -1, 1)))


def test_persistent_errors(gpu):
    scs, ctls = _controllers(True, False)
    batch = drb.controllers.MPPIBatch(ctls)
    with pytest.raises(abi.DrError) as e:
        batch.autotune(3)  # no step yet
    assert e.value.status == abi.DR_ERR_STATE
    with pytest.raises(abi.DrError):
        batch.set_persistent(64, 0, 0)  # more CTAs per SM than fit
    g = H.small_gate(False, K=256, T=40)
    gb = drb.controllers.MPPIBatch([drb.controllers.MPPIController(g.env, g.mppi, g.seed)])
    gb.set_persistent(0, 0, 0)
    with pytest.raises(abi.DrError) as e:
        gb.set_persistent(1, 1, 0)
    assert e.value.status == abi.DR_ERR_UNSUPPORTED
