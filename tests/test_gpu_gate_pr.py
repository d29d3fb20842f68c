"""PR-MPPI on the gate race (dr_gate_prmppi_*) against the reference's own PR-MPPI
kernels compiled for the gate race (USE_ENV_DRONERACE, oracle/_ref gate variant) on
identical injected perturbations and hypotheses, PID action noise off (the reference
draws it from curand): the rollout's running and safety costs of every (plan,
hypothesis, sample), and the candidates' re-check costs."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
import helpers as H

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios


def _case(K=512, T=40, P=8, seed=7, noise=False, agent=0):
    sc = H.small_gate(False, K=K, T=T, seed=seed, noise=noise, agent=agent)
    sc.prmppi = S.make_prmppi(K=K, T=T, P=P)
    return sc


def _noise_thetas(ctl, sc, belief):
    c = sc.prmppi
    n = np.zeros((c.n_timesteps, c.n_samples, 2), np.float32)
    th = np.zeros(c.P, np.int32)
    abi.check(abi.lib().dr_prmppi_debug_noise(ctl.handle, abi.fptr(belief), abi.fptr(n), n.size, abi.iptr(th)), "pr debug_noise")
    return n, th


@pytest.mark.parametrize("K,T,agent,toward", [(512, 40, 0, False), (1000, 64, 1, False), (512, 40, 0, True)])
def test_gate_pr_rollout_matches_reference_kernel(gpu, K, T, agent, toward):
    """toward: the nominal accelerates the ego at the opponent, so that samples collide
    (positive safety costs, terminal states)."""
    sc = _case(K=K, T=T, agent=agent)
    rng = np.random.default_rng(13)
    if toward:
        nominal = np.ascontiguousarray(H.toward_opponent_plan(sc)[0], np.float32).reshape(sc.prmppi.n_timesteps, 2)
    else:
        nominal = rng.normal(0, 1.5, (sc.prmppi.n_timesteps, 2)).astype(np.float32)
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed, nominal=nominal)
    assert ctl.gate
    belief = sc.belief()
    noise, th = _noise_thetas(ctl, sc, belief)
    c = sc.prmppi
    cn = np.zeros((c.P, c.n_samples, 2), np.float32)
    cr = np.zeros_like(cn)
    abi.check(abi.lib().dr_gate_prmppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(cn), abi.fptr(cr)), "gate pr rollout")
    shifted = np.concatenate([nominal[1:], np.zeros((1, 2), np.float32)])
    rcn = np.zeros_like(cn)
    rcr = np.zeros_like(cn)
    rc = O.ref(O.gate_variant_name(False)).refc_pr_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(shifted), O._f(shifted), O._f(noise),
                                                          O._i(th), 9, O._f(rcn), O._f(rcr))
    assert rc == 0
    for name, a, b in (("nom", cn, rcn), ("rob", cr, rcr)):
        mism = ~((a == b) | (np.isnan(a) & np.isnan(b)))
        if not toward:
            assert mism.sum() == 0, f"{name}: {mism.sum()} of {a.size} differ"
        else:
            # near the opponent, the rollouts of the hypothesis whose PID opponent repels
            # the ego differ from the reference's in the last bits (an open finding: the
            # same model in the MPPI rollout matches bit for bit)
            fin = np.isfinite(a) & np.isfinite(b)
            rel = np.abs(a.astype(np.float64) - b)[fin] / np.maximum(1.0, np.abs(b[fin]))
            print(f"{name}: {mism.sum()} of {a.size} differ, hypotheses {sorted(set(th[np.argwhere(mism)[:, 0]].tolist()))}, max rel {rel.max():.2e}")
            assert rel.max() <= 1e-4
    # the comparison covers running costs with boundary terms and positive safety costs
    frac = float(np.mean(cn[..., 1] > 0))
    print("safety > 0 fraction", frac, "running cost range", float(cn[..., 0].min()), float(cn[..., 0].max()))
    if toward:
        assert frac > 0.05


def test_gate_pr_steps(gpu):
    """Closed-loop-style steps through dr_gate_prmppi_step: finite actions within the
    acceleration limit, plans and decisions that move, and a strategic-race call refused."""
    sc = _case(K=1024, T=40, noise=True)
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed)
    ctl.engine = object()
    acts = []
    for _ in range(4):
        a = ctl.getControl(sc.state)
        assert np.all(np.isfinite(a)) and np.linalg.norm(a) <= float(sc.env.max_accel[int(sc.env.i_mppi)]) * 1.0001
        acts.append(a)
        assert ctl.info.cand_cost[0] == ctl.info.cand_cost[0]
    assert np.abs(np.stack(acts)).max() > 0
    with pytest.raises(abi.DrError):
        abi.check(abi.lib().dr_prmppi_step(ctl.handle, C.byref(abi.dr_sim_state()), abi.fptr(ctl.h_belief), abi.fptr(np.zeros(2, np.float32)),
                                           C.byref(ctl.info)), "dr_prmppi_step")
