"""The PyTorch FP64 autograd transcription of the gradient path's objective
(oracle/torch_model.py) against the forward-mode dual-number oracle
(oracle/port/grad.cpp): the same objective value, and the reverse-mode gradient dotted
with random directions equal to the dual number's directional derivative. Two FP64
references built on different differentiation modes that agree pin each other; the GPU
adjoint is checked against both (tests/test_gpu_grad.py)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import O
import helpers as H
from oracle import torch_model as TM


def _case(spl: bool, seed: int, T: int = 40, crash: bool = False, conf: float | None = None):
    sc = H.small_mppi(spl, K=256, T=T, M=8, n_verif=256, seed=7, noise=False)
    if conf is not None:
        # distinguishable hypotheses (a slower second opponent model), so that the belief
        # commits within the horizon and the rollout branches
        sc.env.opp_configs[1].speed_scale[0] = 0.6
        sc.mppi.min_confidence = conf
    c = sc.mppi
    rng = np.random.default_rng(seed)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2))
    if crash:
        U[..., 1] += 3.0  # full sideways push: the rollouts end early (lose)
    w6 = np.array([c.boundary_cost, c.outside_cost, c.win_cost, c.opp_win_cost, c.final_adv_weight, 10.0], np.float64)
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    B = O.spline_matrix(c) if spl else None
    return sc, c, rng, U, w6, belief, B


@pytest.mark.parametrize("spl,seed,crash,conf", [(True, 1, False, None), (False, 2, False, None), (True, 3, True, None), (False, 4, True, None),
                                                 (True, 5, False, 0.8), (False, 6, False, 0.8)])
def test_torch_autograd_matches_dual_oracle(spl, seed, crash, conf):
    sc, c, rng, U, w6, belief, B = _case(spl, seed, crash=crash, conf=conf)
    J, gU, gW = TM.nominal_grad(sc.env, c, sc.state, belief, U, w6, B)
    J64, _, sig = O.nominal_cost(sc, sc.state, belief, U, w6=w6, B=B)
    assert abs(J - J64) <= 1e-12 * max(1.0, abs(J64)), (J, J64)
    gnorm = np.sqrt((gU ** 2).sum() + (gW ** 2).sum())
    assert gnorm > 0
    for _ in range(4):
        dU = rng.normal(0, 1, U.shape)
        dW = rng.normal(0, 1, 6)
        _, dJ, _ = O.nominal_cost(sc, sc.state, belief, U, w6=w6, dU=dU, dW=dW, B=B)
        mine = float((gU * dU).sum() + (gW * dW).sum())
        assert abs(mine - dJ) <= 1e-9 * max(1.0, gnorm * np.sqrt((dU ** 2).sum() + (dW ** 2).sum())), (mine, dJ)
    print(f"spl={spl} crash={crash} conf={conf}: J={J:.6g} |g|={gnorm:.4g} steps/pred/branch {sig.tolist()}")
    if crash:
        assert (sig[:, 0] < c.n_timesteps).any()  # some rollout did end early
    if conf is not None:
        assert (sig[:, 1] > 0).any()  # some rollout did commit to a hypothesis
