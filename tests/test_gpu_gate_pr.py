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
        assert mism.sum() == 0, f"{name}: {mism.sum()} of {a.size} differ"
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


@pytest.mark.parametrize("toward,scale", [(False, 1.5), (True, 0.0)])
def test_gate_pr_step_matches_reference_kernels(gpu, toward, scale):
    """One PR-MPPI control step on the gate race against the reference's kernels built for
    the gate race, PID noise off: the rollout costs (PRMPPIfullRolloutKernel), the cost
    averaging, the three minima and weighted averages (PRMPPIcostAvgKernel,
    PRMPPIcomputeMinCostsKernel, PRMPPIWeightedAverageKernel, prmppi_kernels.cu:134-282)
    and the candidates' costs and safety re-check (PRMPPIcomputeCandidateCostKernel,
    PRMPPIcomputeSafeCostKernel, :285-393) with the host choice of prmppi_controller.cu:
    236-275. Minima identical, plans, nu and candidate costs within 1e-5 relative, the
    candidate choice and useNomPlan equal. toward: the nominal drives the ego at the PID
    opponent, so that the hypothesis following the other raceline meets it."""
    RTOL, ATOL = 1e-5, 1e-6
    sc = _case(K=1000, T=40, agent=0)
    c = sc.prmppi
    T, K, P = c.n_timesteps, c.n_samples, c.P
    if toward:
        nominal = np.ascontiguousarray(H.toward_opponent_plan(sc)[0], np.float32).reshape(T, 2)
    else:
        nominal = np.random.default_rng(17).normal(0, scale, (T, 2)).astype(np.float32)
    belief = sc.belief()
    probe = drb.controllers.PRMPPIController(sc.env, c, sc.seed, nominal=nominal)
    noise, th = _noise_thetas(probe, sc, belief)
    cn = np.zeros((P, K, 2), np.float32)
    cr = np.zeros_like(cn)
    abi.check(abi.lib().dr_gate_prmppi_debug_rollout(probe.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(cn), abi.fptr(cr)), "gate pr rollout")
    shifted = np.concatenate([nominal[1:], np.zeros((1, 2), np.float32)])
    variant = O.gate_variant_name(False)
    rcn, rcr = np.zeros_like(cn), np.zeros_like(cn)
    rc = O.ref(variant).refc_pr_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(shifted), O._f(shifted), O._f(noise), O._i(th), 9,
                                        O._f(rcn), O._f(rcr))
    assert rc == 0
    same = ((cn == rcn) | (np.isnan(cn) & np.isnan(rcn))) & ((cr == rcr) | (np.isnan(cr) & np.isnan(rcr)))
    assert same.all(), f"{(~same).sum()} rollout costs differ"
    lam = np.full(3, c.inv_temperature, np.float32)
    mins = np.zeros(3, np.float32)
    c1, c2, nr = (np.zeros((T, 2), np.float32) for _ in range(3))
    nu = np.zeros(3, np.float32)
    rc = O.ref(variant).refc_pr_update(C.byref(c), O._f(rcn.copy()), O._f(rcr.copy()), O._f(noise), O._f(shifted), O._f(shifted), O._f(lam), O._f(mins),
                                       O._f(c1), O._f(c2), O._f(nr), O._f(nu))
    assert rc == 0
    cand = np.zeros(2 * P, np.float32)
    safe = np.zeros(P, np.float32)
    rc = O.ref(variant).refc_pr_candidates(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(c1), O._f(c2), O._f(c1), O._i(th), 5, O._f(cand),
                                           O._f(safe))
    assert rc == 0
    m1 = np.float32(np.sum(cand[:P], dtype=np.float32)) / np.float32(P)
    m2 = np.float32(np.sum(cand[P:], dtype=np.float32)) / np.float32(P)
    reset = bool(m2 < m1)
    chosen = c1 if m1 <= m2 else c2
    if not m1 <= m2:
        rc = O.ref(variant).refc_pr_candidates(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(c1), O._f(c2), O._f(c2), O._i(th), 5, O._f(cand),
                                               O._f(safe))
        assert rc == 0
    use_nom = not np.any(safe > 0.0)
    ctl = drb.controllers.PRMPPIController(sc.env, c, sc.seed, nominal=nominal)
    ctl.engine = object()
    action = ctl.getControl(sc.state)
    info = ctl.info
    assert np.array_equal(np.array(info.min_costs, np.float32), mins), (np.array(info.min_costs), mins)
    np.testing.assert_allclose(np.array(info.nu, np.float32), nu, rtol=RTOL)
    np.testing.assert_allclose(np.array(info.cand_cost, np.float32), [m1, m2], rtol=RTOL)
    assert bool(info.reset_nom) == reset
    assert bool(info.use_nom_plan) == use_nom
    nom, rob = ctl.nominals()
    np.testing.assert_allclose(nom.reshape(T, 2), chosen, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(rob.reshape(T, 2), nr, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(action, (chosen if use_nom else nr)[0], rtol=RTOL, atol=ATOL)
    print(f"toward {toward}: choice {'cand2' if reset else 'cand1'}, useNomPlan {use_nom}, candidate costs {m1:.6g} / {m2:.6g}, "
          f"plans bit-identical {np.mean(nom.reshape(T, 2) == chosen):.3f} / {np.mean(rob.reshape(T, 2) == nr):.3f}")
