"""Gradient path on the GPU (grad_kernels.cu through dr_mppi_nominal_grad and the torch
op): the adjoint kernel's gradients against the FP64 forward-mode reference
(oracle/port/grad.cpp) on 32 random directions, checkpoint-stride invariance, batching,
the autograd face, and the refinement step inside the control step."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from conftest import O, drb
import helpers as H

pytestmark = pytest.mark.gpu

abi = drb.abi


def _grad_mod():
    return importlib.import_module("drone_race_b200.grad")


def _torch():
    import torch

    return torch


def _weights(c, final_opp=10.0):
    return np.array([c.boundary_cost, c.outside_cost, c.win_cost, c.opp_win_cost, c.final_adv_weight, final_opp], np.float32)


def _kernel(ctl, sc, belief, U, w6, ckpt=0):
    torch = _torch()
    G = _grad_mod()
    Ut = torch.tensor(np.asarray(U, np.float32)).reshape(-1, *U.shape[-3:]).cuda()
    Wt = torch.tensor(np.asarray(w6, np.float32)).reshape(-1, 6).expand(Ut.shape[0], 6).contiguous().cuda()
    J, dU, dW = G.nominal_cost_grad(int(ctl.handle.value), G._state_bytes(sc.state), torch.tensor(belief), Ut, Wt, True, ckpt)
    torch.cuda.synchronize()
    return J.cpu().numpy(), dU.cpu().numpy(), dW.cpu().numpy()


@pytest.mark.parametrize("spl", [True, False])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_gradient_matches_fp64_reference(gpu, spl, seed):
    sc = H.small_mppi(spl, K=256, T=40)
    c = sc.mppi
    ctl = H.mppi_ctl(sc)
    rng = np.random.default_rng(seed)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2)).astype(np.float32)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w6 = _weights(c)
    J, dU, dW = _kernel(ctl, sc, belief, U, w6)
    J64, _, _ = O.nominal_cost(sc, sc.state, belief, U.astype(np.float64), w6=w6.astype(np.float64))
    assert abs(J[0] - J64) <= 1e-4 * max(1.0, abs(J64)), (J[0], J64)
    gnorm = np.sqrt((dU[0].astype(np.float64) ** 2).sum() + (dW[0].astype(np.float64) ** 2).sum())
    errs = []
    for _ in range(32):
        d = rng.normal(0, 1, U.shape)
        d /= np.linalg.norm(d)
        dw = rng.normal(0, 1, 6)
        dw /= np.linalg.norm(dw)
        _, jvp, _ = O.nominal_cost(sc, sc.state, belief, U.astype(np.float64), w6=w6.astype(np.float64), dU=d, dW=dw)
        mine = float((dU[0].astype(np.float64) * d).sum() + (dW[0].astype(np.float64) * dw).sum())
        errs.append(abs(mine - jvp) / gnorm)
    errs = np.array(errs)
    print(f"spl={spl} seed={seed} J={J[0]:.6g} |g|={gnorm:.4g} err median {np.median(errs):.2e} max {errs.max():.2e}")
    # FP32 forward and adjoint against FP64: directional derivatives agree to 1e-3 of |g|
    assert np.median(errs) < 1e-4 and errs.max() < 1e-3, errs


@pytest.mark.parametrize("spl", [True, False])
@pytest.mark.parametrize("seed", [11, 12])
def test_gradient_matches_torch_fp64_autograd(gpu, spl, seed):
    """The whole gradient (controls and weights) against the PyTorch FP64 autograd
    transcription of the objective (oracle/torch_model.py, reverse mode)."""
    from oracle import torch_model as TM

    sc = H.small_mppi(spl, K=256, T=40)
    c = sc.mppi
    ctl = H.mppi_ctl(sc)
    rng = np.random.default_rng(seed)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2)).astype(np.float32)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w6 = _weights(c)
    J, dU, dW = _kernel(ctl, sc, belief, U, w6)
    B = O.spline_matrix(c) if spl else None
    J64, gU, gW = TM.nominal_grad(sc.env, c, sc.state, belief, U.astype(np.float64), w6.astype(np.float64), B)
    assert abs(J[0] - J64) <= 1e-4 * max(1.0, abs(J64)), (J[0], J64)
    g64 = np.concatenate([gU.ravel(), gW])
    g32 = np.concatenate([dU[0].ravel(), dW[0]]).astype(np.float64)
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"spl={spl} seed={seed}: |g|={np.linalg.norm(g64):.4g}, |g32 - g64| / |g64| = {rel:.2e}")
    # FP32 forward and adjoint against the FP64 reverse-mode gradient: 2e-3 of |g|
    assert rel < 2e-3, rel


def test_checkpoint_stride_does_not_change_the_result(gpu):
    sc = H.small_mppi(True, K=256, T=40)
    ctl = H.mppi_ctl(sc)
    rng = np.random.default_rng(4)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(sc.mppi), 2)).astype(np.float32)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w6 = _weights(sc.mppi)
    ref = _kernel(ctl, sc, belief, U, w6, ckpt=1)
    for ck in (0, 2, 7, 13, 40):
        out = _kernel(ctl, sc, belief, U, w6, ckpt=ck)
        for a, b in zip(ref, out):
            assert np.array_equal(a, b), ck


def test_batch_of_start_points_equals_single_calls(gpu):
    sc = H.small_mppi(False, K=256, T=40)
    ctl = H.mppi_ctl(sc)
    rng = np.random.default_rng(6)
    U = rng.normal(0, 0.7, (5, sc.n_theta + 1, O.mk(sc.mppi), 2)).astype(np.float32)
    W = np.stack([_weights(sc.mppi) * (1 + 0.1 * i) for i in range(5)])
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    J, dU, dW = _kernel(ctl, sc, belief, U, W)
    for i in range(5):
        Ji, dUi, dWi = _kernel(ctl, sc, belief, U[i], W[i])
        assert J[i] == Ji[0] and np.array_equal(dU[i], dUi[0]) and np.array_equal(dW[i], dWi[0])


def test_autograd_backward_is_the_adjoint(gpu):
    torch = _torch()
    G = _grad_mod()
    sc = H.small_mppi(True, K=256, T=40)
    ctl = H.mppi_ctl(sc)
    rng = np.random.default_rng(8)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(sc.mppi), 2)).astype(np.float32)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w6 = _weights(sc.mppi)
    Ut = torch.tensor(U, device="cuda", requires_grad=True)
    Wt = torch.tensor(w6, device="cuda", requires_grad=True)
    J = G.nominal_cost(ctl, sc.state, belief, Ut, Wt)
    (3.0 * J).backward()
    J0, dU, dW = _kernel(ctl, sc, belief, U, w6)
    assert float(J.detach()) == J0[0]
    assert np.array_equal(Ut.grad.cpu().numpy(), 3.0 * dU[0])
    assert np.array_equal(Wt.grad.cpu().numpy(), 3.0 * dW[0])


@pytest.mark.parametrize("spl", [True, False])
def test_refinement_keeps_the_best_plan(gpu, spl):
    torch = _torch()
    G = _grad_mod()
    sc = H.small_mppi(spl, K=512, T=40)
    plain = H.mppi_ctl(sc)
    ref = H.mppi_ctl(sc)
    ref.set_grad_refine(3, 0.05, 0)
    for ctl in (plain, ref):
        ctl.engine = object()
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    improved = 0
    for k in range(6):
        a_plain = plain.getControl(sc.state)
        kn_plain = plain.knots()
        ref.getControl(sc.state)
        info = ref.info
        assert info.grad_best_step >= 0
        assert info.grad_cost_refined <= info.grad_cost_plain
        # the refinement starts from the plain update: same objective as the plain
        # controller's plan (both controllers have seen the same steps so far only while
        # the refined one kept the plain plan)
        kn_ref = ref.knots()
        Jr = G.nominal_cost(ref, sc.state, belief, torch.tensor(kn_ref, device="cuda"))
        assert float(Jr) == info.grad_cost_refined
        if info.grad_best_step == 0:
            assert np.array_equal(kn_ref, kn_plain)
        else:
            improved += 1
            Jp = G.nominal_cost(ref, sc.state, belief, torch.tensor(kn_plain, device="cuda"))
            assert float(Jp) == info.grad_cost_plain
            break
        del a_plain
    assert improved >= 1


def test_errors(gpu):
    sc = H.small_mppi(True, K=256, T=40)
    ctl = H.mppi_ctl(sc)
    with pytest.raises(abi.DrError):
        ctl.set_grad_refine(abi.DR_GRAD_MAX_STEPS + 1)
    with pytest.raises(abi.DrError):
        ctl.set_grad_refine(2, 0.0)
    with pytest.raises(abi.DrError):
        ctl.set_grad_refine(2, 0.05, 41)
    g = H.small_gate(False, K=256, T=40)
    gctl = drb.controllers.MPPIController(g.env, g.mppi, g.seed)
    with pytest.raises(abi.DrError) as e:
        gctl.set_grad_refine(2)
    assert e.value.status == abi.DR_ERR_UNSUPPORTED


def test_uneven_batch_with_refinement_equals_single_controllers(gpu):
    """Controllers of different sample counts, horizons and verification sizes, some with
    gradient refinement, stepped as one batch (one launch per kernel over a tile table,
    graph-replayed, verification overlapped) act exactly as when stepped alone."""
    S = drb.scenarios
    sizes = [(256, 32, 256, 0), (1024, 48, 512, 3), (512, 64, 1024, 2)]
    scs = [S.circle_race(agent=a, K=k, T=t, n_verif=v) for a, (k, t, v, _) in enumerate(sizes)]
    singles = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    batched = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    for (_, _, _, g), c1, c2 in zip(sizes, singles, batched):
        if g:
            c1.set_grad_refine(g, 0.05, 0)
            c2.set_grad_refine(g, 0.05, 0)
        c1.engine = object()
    batch = drb.controllers.MPPIBatch(batched)
    beliefs = np.stack([s.belief() for s in scs])
    for _ in range(3):
        a1 = np.stack([c.getControl(s.state) for c, s in zip(singles, scs)])
        a2 = batch.step([s.state for s in scs], beliefs)
        assert np.array_equal(a1, a2)
        for c1, c2 in zip(singles, batched):
            assert np.array_equal(c1.h_nominal, c2.h_nominal)


def _multi_scenario(nopp: int, nth: int, spl: bool):
    """Small strategic race with nopp opponents and nth distinguishable hypotheses."""
    S = drb.scenarios
    r = 0.4
    grids = drb.track.track_grids(drb.track.circle_track(6.0))
    kinds = [("insensitive", "default"), ("insensitive", "no-block"), ("default", "default"), ("conservative", "no-block")]
    configs = []
    for th in range(nth):
        s1, s3 = kinds[th % 4]
        p = S.opp_preset(r, s1=s1, s3=s3, speed_scale=0.8 + 0.4 * th / max(nth - 1, 1))
        configs.append([p] * nopp)
    env = S.make_env(grids, n_opp=nopp, opp_configs=configs, dt=0.1, drone_radius=r, max_speed=[3, 2, 2, 2], max_accel=[2, 3, 3, 3],
                     track_width=2.0, kV=5.0, max_opp_lat_dist_fact=1.9)
    idx = [int(v) for v in np.round(np.linspace(0.05, 0.2, nopp + 1) * 512)]
    st = S.initial_state(grids, idx, nopp)
    sc = S.Scenario(env=env, grids=grids, state=st, name=f"multi_{nopp}_{nth}")
    sc.mppi = S.make_mppi(K=256, T=40, use_splines=spl, M=10, n_verif_samples=512, verif_horizon=30, final_opp_adv_weight=20.0)
    return sc


@pytest.mark.parametrize("nopp,nth", [(2, 2), (1, 4), (1, 8), (1, 1)])
def test_gradient_matches_fp64_reference_other_sizes(gpu, nopp, nth):
    """The other compiled (n_opp, n_theta) combinations: two opponents, and 1, 4 and 8
    hypotheses (clusters of up to 8 CTAs)."""
    sc = _multi_scenario(nopp, nth, True)
    c = sc.mppi
    ctl = drb.controllers.MPPIController(sc.env, c, 17)
    rng = np.random.default_rng(nopp * 10 + nth)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2)).astype(np.float32)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w6 = _weights(c, final_opp=20.0)
    J, dU, dW = _kernel(ctl, sc, belief, U, w6)
    J64, _, _ = O.nominal_cost(sc, sc.state, belief, U.astype(np.float64), w6=w6.astype(np.float64))
    assert abs(J[0] - J64) <= 1e-4 * max(1.0, abs(J64)), (J[0], J64)
    gnorm = np.sqrt((dU[0].astype(np.float64) ** 2).sum() + (dW[0].astype(np.float64) ** 2).sum())
    errs = []
    for _ in range(16):
        d = rng.normal(0, 1, U.shape)
        d /= np.linalg.norm(d)
        dw = rng.normal(0, 1, 6)
        dw /= np.linalg.norm(dw)
        _, jvp, _ = O.nominal_cost(sc, sc.state, belief, U.astype(np.float64), w6=w6.astype(np.float64), dU=d, dW=dw)
        errs.append(abs(float((dU[0].astype(np.float64) * d).sum() + (dW[0].astype(np.float64) * dw).sum()) - jvp) / gnorm)
    errs = np.array(errs)
    print(f"nopp={nopp} nth={nth} J={J[0]:.6g} |g|={gnorm:.4g} err median {np.median(errs):.2e} max {errs.max():.2e}")
    assert np.median(errs) < 1e-4 and errs.max() < 1e-3, errs
