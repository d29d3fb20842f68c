"""Parity at the benchmark's own configurations, against the reference's own CUDA kernels
(compiled from the reference sources into oracle/_ref) on identical injected
perturbations and hypotheses, in-rollout noise off (the reference draws it from curand).

* MPPI, the headline workload: each of the four circle_race agents (K 4096, H 64, dense
  controls, 2 hypotheses): rollout costs and branch records bit-identical to
  fullRolloutKernel (kernels.cu:34-171), per-branch costs identical to
  aggregateBranchCostsKernel (kernels.cu:175-217), and the update's minima identical and
  its controls within 1e-5 relative to computeMaskedMinCostsKernel +
  weightedAverageKernelUnified + clampNominalKernel (kernels.cu:221-456).
* PR-MPPI: the cost averaging, the three minima and the three weighted averages
  (PRMPPIcostAvgKernel, PRMPPIcomputeMinCostsKernel, PRMPPIWeightedAverageKernel,
  prmppi_kernels.cu:134-282) and the candidate choice and safety decision
  (PRMPPIcomputeCandidateCostKernel, PRMPPIcomputeSafeCostKernel, prmppi_kernels.cu:
  285-393, with the host choice of prmppi_controller.cu:236-275), on a small case and on
  the benchmark's PR configuration (8 hypotheses, P 8, K 2048, H 64): minima identical,
  candidates, new robust plan, nu and candidate costs within 1e-5 relative, candidate
  choice and useNomPlan equal.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
from helpers import zero_env_noise

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios

RTOL, ATOL = 1e-5, 1e-6  # "within 1e-5 relative" (atol only for entries at zero)


def _dev_noise(ctl, sc):
    c = sc.mppi
    n = np.zeros((sc.n_theta + 1, O.mk(c), c.n_samples, 2), np.float32)
    abi.check(abi.lib().dr_mppi_debug_noise(ctl.handle, abi.fptr(n), n.size), "debug_noise")
    return n


@pytest.mark.parametrize("agent", [0, 1, 2, 3])
def test_headline_config_rollout_and_update_match_reference(gpu, agent):
    sc = S.circle_race(agent=agent, seed=0, K=4096, T=64, use_splines=False, n_theta=2, n_verif=2**17)
    zero_env_noise(sc)
    c = sc.mppi
    K, T, nth = c.n_samples, c.n_timesteps, sc.n_theta
    nbp = nth + 1
    # a plan accelerating the ego at the opponent (4 m/s^2): the opponent's reaction splits
    # the hypotheses, so most samples commit to a branch, and some collide
    st = sc.state
    d = np.array([st.pos[2] - st.pos[0], st.pos[3] - st.pos[1]], np.float64)
    nominal = np.broadcast_to(d / np.linalg.norm(d) * 4.0, (nbp, T, 2)).astype(np.float32).copy()
    ctl = drb.controllers.MPPIController(sc.env, c, sc.seed, nominal=nominal)
    belief = sc.belief()
    noise = _dev_noise(ctl, sc)
    ct = np.zeros((nth, K), np.float32)
    bu = np.zeros((nth, K), np.int32)
    bt = np.zeros((nth, K), np.int32)
    costs = np.zeros((nbp, K), np.float32)
    abi.check(abi.lib().dr_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(ct), abi.iptr(bu), abi.iptr(bt),
                                              abi.fptr(costs)), "debug_rollout")
    kn = ctl.knots().copy()
    variant = O.ref_variant_name(2, False)
    rct, rbu, rbt = np.zeros_like(ct), np.zeros_like(bu), np.zeros_like(bt)
    B = np.zeros(1, np.float32)
    rc = O.ref(variant).refc_mppi_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(belief), O._f(np.ascontiguousarray(kn)), O._f(noise),
                                          O._f(B), 123, O._f(rct), O._i(rbu), O._i(rbt))
    assert rc == 0
    assert np.array_equal(bu, rbu) and np.array_equal(bt, rbt)
    same = (ct == rct) | (np.isnan(ct) & np.isnan(rct))
    assert same.all(), f"{(~same).sum()} of {ct.size} rollout costs differ"
    # the case must exercise the belief update and the branch bookkeeping
    assert np.mean(bu != 0) > 0.5
    # update on these rollout outputs: ours (debug hook) and the reference's kernels
    dense = np.zeros((nbp, T, 2), np.float32)
    mins = np.zeros((nbp, T), np.float32)
    nu = np.zeros(nbp, np.float32)
    abi.check(abi.lib().dr_mppi_debug_update(ctl.handle, abi.fptr(belief), abi.fptr(ct), abi.iptr(bu), abi.iptr(bt), abi.fptr(dense), abi.fptr(mins),
                                             abi.fptr(nu)), "debug_update")
    r_kn = kn.copy()
    r_dense = np.zeros_like(dense)
    r_mins = np.zeros_like(mins)
    r_nu = np.zeros_like(nu)
    r_costs = np.zeros_like(costs)
    rc = O.ref(variant).refc_mppi_update(C.byref(sc.env), C.byref(c), O._f(belief), O._f(rct), O._i(rbu), O._i(rbt), O._f(noise), O._f(B), O._f(r_kn),
                                         O._f(r_dense), O._f(r_mins), O._f(r_nu), O._f(r_costs))
    assert rc == 0
    assert np.array_equal(costs, r_costs)
    assert np.array_equal(mins, r_mins)
    np.testing.assert_allclose(nu, r_nu, rtol=RTOL)
    np.testing.assert_allclose(dense, r_dense, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(ctl.knots(), r_kn, rtol=RTOL, atol=ATOL)
    print(f"agent {agent}: samples that branched {np.mean(bu != 0):.3f}, cost range {np.ptp(ct[np.isfinite(ct)]):.4g}; "
          f"updated controls bit-identical {np.mean(dense == r_dense):.4f}")


def _pr_case(nth, K, T):
    if nth == 2:
        sc = S.strat_race(use_pr=True, K=K, T=T)
        sc.prmppi = S.make_prmppi(K=K, T=T, P=8)
    else:
        sc = S.robust_race(agent=0, seed=3, K=K, T=T, P=8, n_theta=nth)
    return zero_env_noise(sc)


@pytest.mark.parametrize("nth,K,T,scale", [(2, 512, 40, 0.8), (8, 2048, 64, 0.8), (8, 2048, 64, 2.5)])
def test_pr_update_and_candidates_match_reference(gpu, nth, K, T, scale):
    sc = _pr_case(nth, K, T)
    c = sc.prmppi
    P = c.P
    rng = np.random.default_rng(40 + nth + int(10 * scale))
    nominal = rng.normal(0, scale, (T, 2)).astype(np.float32)
    belief = sc.belief()
    probe = drb.controllers.PRMPPIController(sc.env, c, sc.seed, nominal=nominal)
    noise = np.zeros((T, K, 2), np.float32)
    th = np.zeros(P, np.int32)
    abi.check(abi.lib().dr_prmppi_debug_noise(probe.handle, abi.fptr(belief), abi.fptr(noise), noise.size, abi.iptr(th)), "pr debug_noise")
    cn = np.zeros((P, K, 2), np.float32)
    cr = np.zeros_like(cn)
    abi.check(abi.lib().dr_prmppi_debug_rollout(probe.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(cn), abi.fptr(cr)), "pr debug_rollout")
    # the reference's update on the same rollout costs, perturbation and shifted nominals
    shifted = np.concatenate([nominal[1:], np.zeros((1, 2), np.float32)])
    lam = np.full(3, c.inv_temperature, np.float32)
    mins = np.zeros(3, np.float32)
    c1, c2, nr = (np.zeros((T, 2), np.float32) for _ in range(3))
    nu = np.zeros(3, np.float32)
    variant = O.ref_variant_name(nth, True)
    rc = O.ref(variant).refc_pr_update(C.byref(c), O._f(cn.copy()), O._f(cr.copy()), O._f(noise), O._f(shifted), O._f(shifted), O._f(lam), O._f(mins),
                                       O._f(c1), O._f(c2), O._f(nr), O._f(nu))
    assert rc == 0
    # the reference's candidate costs, its host choice and its safety check of the choice
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
    # one control step of an identical controller
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
    print(f"nth {nth} K {K}: choice {'cand2' if reset else 'cand1'}, useNomPlan {use_nom}, plans bit-identical "
          f"{np.mean(nom.reshape(T, 2) == chosen):.3f} / {np.mean(rob.reshape(T, 2) == nr):.3f}")
