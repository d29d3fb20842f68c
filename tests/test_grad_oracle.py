"""The FP64 reference of the gradient path (oracle/port/grad.cpp): the directional
derivative its forward-mode dual number gives equals central finite differences of its
value (epsilon 1e-3 on 32 random directions in control and cost-weight space) wherever
the rollout is smooth within the difference, the check the CUDA adjoint is held to."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import O
import helpers as H


def _weights(c, final_opp=10.0):
    return np.array([c.boundary_cost, c.outside_cost, c.win_cost, c.opp_win_cost, c.final_adv_weight, final_opp], np.float64)


def _fd_check(sc, U, w6, belief, rng, n_dir=32, eps=1e-3):
    """Returns (relative errors on the smooth directions, number of non-smooth ones)."""
    def val(du, dw, e):
        return O.nominal_cost(sc, sc.state, belief, U + e * du, w6=w6 + e * dw)[0]

    rels, rough = [], 0
    for _ in range(n_dir):
        d = rng.normal(0, 1, U.shape)
        d /= np.linalg.norm(d)
        dw = rng.normal(0, 1, 6)
        dw /= np.linalg.norm(dw)
        _, jvp, _ = O.nominal_cost(sc, sc.state, belief, U, w6=w6, dU=d, dW=dw)
        f1 = (val(d, dw, eps) - val(d, dw, -eps)) / (2 * eps)
        f2 = (val(d, dw, eps / 4) - val(d, dw, -eps / 4)) / (eps / 2)
        # a discrete decision (projection segment, branch time, clamp) inside +-eps shows
        # as two differences that disagree; those directions are not comparable
        if abs(f1 - f2) > 1e-5 * max(abs(f1), abs(f2), 1e-9):
            rough += 1
            continue
        rels.append(abs(f1 - jvp) / max(abs(jvp), abs(f1), 1e-12))
    return np.array(rels), rough


@pytest.mark.parametrize("spl", [True, False])
@pytest.mark.parametrize("seed", [1, 3])
def test_jvp_matches_central_differences(spl, seed):
    sc = H.small_mppi(spl, K=256, T=40)
    c = sc.mppi
    rng = np.random.default_rng(seed)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2))
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    rels, rough = _fd_check(sc, U, _weights(c), belief, rng)
    assert rough <= 4, rough
    assert len(rels) >= 28
    assert rels.max() < 1e-6, rels.max()


def test_jvp_across_a_branch_commitment():
    """Two distinguishable opponent hypotheses from an even belief: every rollout commits
    to a branch plan a few steps in, and the derivative follows the switch of plans."""
    sc = H.small_mppi(True, K=256, T=40)
    c = sc.mppi
    sc.env.opp_configs[1].speed_scale[0] = 0.6
    c.min_confidence = 0.8
    belief = np.array([0.5, 0.5], np.float32)
    rng = np.random.default_rng(1)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2))
    _, _, sig = O.nominal_cost(sc, sc.state, belief, U, w6=_weights(c))
    assert (sig[:, 1] > 0).any(), sig  # a commitment happened
    rels, rough = _fd_check(sc, U, _weights(c), belief, rng, n_dir=16)
    assert rough <= 3 and len(rels) >= 13
    assert rels.max() < 1e-6, rels.max()


def test_weight_gradient_is_the_cost_features():
    """J is linear in the six weights: J(w) = J(0-weights) + sum_i w_i dJ/dw_i."""
    sc = H.small_mppi(False, K=256, T=40)
    c = sc.mppi
    rng = np.random.default_rng(2)
    U = rng.normal(0, 0.7, (sc.n_theta + 1, O.mk(c), 2))
    belief = np.array(sc.env.init_belief[: sc.n_theta], np.float32)
    w = _weights(c)
    J, _, _ = O.nominal_cost(sc, sc.state, belief, U, w6=w)
    g = np.array([O.nominal_cost(sc, sc.state, belief, U, w6=w, dW=np.eye(6)[i])[1] for i in range(6)])
    assert abs(float(g @ w) - J) <= 1e-9 * max(1.0, abs(J))
