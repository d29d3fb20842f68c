"""MPPI parity on the B200: the CUDA path against the reference's own CUDA kernels
(compiled from the reference sources into oracle/_ref) on identical injected
perturbations, and against the CPU oracle port in FP32 and FP64."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
from helpers import OracleMPPI, mppi_ctl, random_nominal, small_mppi, zero_env_noise

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios


def _dev_rollout(ctl, sc, belief):
    K, nth = sc.mppi.n_samples, sc.n_theta
    ct = np.zeros((nth, K), np.float32)
    bu = np.zeros((nth, K), np.int32)
    bt = np.zeros((nth, K), np.int32)
    costs = np.zeros((nth + 1, K), np.float32)
    abi.check(abi.lib().dr_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(ct), abi.iptr(bu), abi.iptr(bt),
                                              abi.fptr(costs)), "debug_rollout")
    return ct, bu, bt, costs


def _dev_noise(ctl, sc):
    c = sc.mppi
    n = np.zeros((sc.n_theta + 1, O.mk(c), c.n_samples, 2), np.float32)
    abi.check(abi.lib().dr_mppi_debug_noise(ctl.handle, abi.fptr(n), n.size), "debug_noise")
    return n


@pytest.mark.parametrize("spl", [True, False])
def test_noise_bit_exact(gpu, spl):
    sc = small_mppi(spl, K=300)
    ctl = mppi_ctl(sc)
    assert np.array_equal(_dev_noise(ctl, sc), O.mppi_noise(sc, 0))


@pytest.mark.parametrize("spl", [True, False])
def test_rollout_matches_reference_kernel(gpu, spl):
    """fullRolloutKernel (kernels.cu:34-171) vs the fused rollout, same perturbation:
    per-sample costs and branch bookkeeping must be identical."""
    variant = O.ref_variant_name(2, spl)
    sc = small_mppi(spl, K=1024, T=40, noise=False)
    rng = np.random.default_rng(1)
    nominal = random_nominal(sc, rng)
    ctl = mppi_ctl(sc, nominal=nominal)
    belief = sc.belief()
    if spl:
        # one full step first, so that the knots are no longer the initial zeros
        ctl.engine = object()
        ctl.getControl(sc.state)
    noise = _dev_noise(ctl, sc)
    ct, bu, bt, costs = _dev_rollout(ctl, sc, belief)
    kn = ctl.knots()  # the (shifted) knots the rollout used
    assert np.abs(kn).max() > 0
    rct = np.zeros_like(ct)
    rbu = np.zeros_like(bu)
    rbt = np.zeros_like(bt)
    B = O.spline_matrix(sc.mppi) if spl else np.zeros(1, np.float32)
    rc = O.ref(variant).refc_mppi_rollout(C.byref(sc.env), C.byref(sc.mppi), C.byref(sc.state), O._f(belief), O._f(np.ascontiguousarray(kn)),
                                          O._f(noise), O._f(B), 123, O._f(rct), O._i(rbu), O._i(rbt))
    assert rc == 0
    assert np.array_equal(bu, rbu) and np.array_equal(bt, rbt)
    mism = ~((ct == rct) | (np.isnan(ct) & np.isnan(rct)))
    assert mism.sum() == 0, f"{mism.sum()} of {ct.size} costs differ; first {np.argwhere(mism)[:5]}"
    # aggregation (aggregateBranchCostsKernel) against the reference's own update path
    rcosts = np.zeros_like(costs)
    dummy = np.zeros((sc.n_theta + 1) * sc.mppi.n_timesteps * 2, np.float32)
    spl_buf = np.ascontiguousarray(kn).copy()
    mins = np.zeros((sc.n_theta + 1) * O.mk(sc.mppi), np.float32)
    nu = np.zeros(sc.n_theta + 1, np.float32)
    rc = O.ref(variant).refc_mppi_update(C.byref(sc.env), C.byref(sc.mppi), O._f(belief), O._f(rct), O._i(rbu), O._i(rbt), O._f(noise), O._f(B),
                                         O._f(spl_buf), O._f(dummy), O._f(mins), O._f(nu), O._f(rcosts))
    assert rc == 0
    assert np.array_equal(costs, rcosts)


@pytest.mark.parametrize("spl", [True, False])
def test_update_matches_reference_kernels(gpu, spl):
    """masked min + weighted average + interpolation + clamp (kernels.cu:221-456) on the
    same rollout outputs: new knots / dense nominal, minCosts and nu."""
    variant = O.ref_variant_name(2, spl)
    sc = small_mppi(spl, K=1024, T=40, noise=False)
    rng = np.random.default_rng(2)
    ctl = mppi_ctl(sc, nominal=random_nominal(sc, rng))
    belief = np.array([0.3, 0.7], np.float32)
    noise = _dev_noise(ctl, sc)
    kn = ctl.knots().copy()
    B = O.spline_matrix(sc.mppi) if spl else np.zeros(1, np.float32)
    ct, bu, bt = O.mppi_rollout(sc, belief, kn, noise, B if spl else None, 0, prec=32)
    ct32 = ct.astype(np.float32)
    nbp, T, M = sc.n_theta + 1, sc.mppi.n_timesteps, O.mk(sc.mppi)
    dense = np.zeros((nbp, T, 2), np.float32)
    mins = np.zeros((nbp, M), np.float32)
    nu = np.zeros(nbp, np.float32)
    abi.check(abi.lib().dr_mppi_debug_update(ctl.handle, abi.fptr(belief), abi.fptr(ct32), abi.iptr(bu), abi.iptr(bt), abi.fptr(dense), abi.fptr(mins),
                                             abi.fptr(nu)), "debug_update")
    new_kn = ctl.knots()
    r_kn = kn.copy()
    r_dense = np.zeros_like(dense)
    r_mins = np.zeros_like(mins)
    r_nu = np.zeros_like(nu)
    rc = O.ref(variant).refc_mppi_update(C.byref(sc.env), C.byref(sc.mppi), O._f(belief), O._f(ct32), O._i(bu), O._i(bt), O._f(noise), O._f(B),
                                         O._f(r_kn), O._f(r_dense), O._f(r_mins), O._f(r_nu), None)
    assert rc == 0
    assert np.array_equal(mins, r_mins)
    np.testing.assert_allclose(nu, r_nu, rtol=1e-6)
    np.testing.assert_allclose(new_kn, r_kn, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(dense, r_dense, rtol=1e-5, atol=1e-6)
    exact = np.mean(new_kn == r_kn)
    print(f"update bit-exact fraction: {exact:.4f}")


@pytest.mark.parametrize("spl", [True, False])
def test_rollout_matches_oracle_with_env_noise(gpu, spl):
    """With opponent action noise on (Philox streams on both sides), the GPU rollout
    against the FP32 oracle port; disagreements only where the FP32 host/device paths
    differ in rounding (FMA contraction, libm) and a comparison flips."""
    sc = small_mppi(spl, K=1024, T=40, noise=True)
    rng = np.random.default_rng(3)
    ctl = mppi_ctl(sc, nominal=random_nominal(sc, rng))
    belief = sc.belief()
    kn = ctl.knots().copy()
    B = O.spline_matrix(sc.mppi) if spl else None
    noise = O.mppi_noise(sc, 0)
    ct, bu, bt, _ = _dev_rollout(ctl, sc, belief)
    oct32, obu, obt = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=32)
    oct64, _, _ = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=64)
    rel = np.abs(ct - oct32) / np.maximum(1.0, np.abs(oct32))
    close = rel <= 1e-5
    frac = close.mean()
    rel64 = np.abs(ct - oct64) / np.maximum(1.0, np.abs(oct64))
    print(f"fp32 oracle agreement {frac:.4f}; median |gpu-fp64|/|fp64| {np.median(rel64):.2e}")
    assert frac >= 0.97
    assert np.mean(bu == obu) >= 0.97


def test_verification_matches_oracle(gpu):
    sc = small_mppi(False, K=256, T=40, n_verif=4096, noise=True)
    rng = np.random.default_rng(4)
    ctl = mppi_ctl(sc, exact_verify=True)
    plan = random_nominal(sc, rng, 1.0)
    belief = sc.belief()
    fc = np.zeros(sc.mppi.n_timesteps, np.uint32)
    ft = np.zeros(sc.mppi.n_verif_samples, np.int32)
    th = np.zeros(sc.mppi.n_verif_samples, np.int32)
    abi.check(abi.lib().dr_mppi_debug_verify(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(plan), 0, abi.uptr(fc), abi.iptr(ft),
                                             abi.iptr(th)), "debug_verify")
    ofc, oft, oth = O.mppi_verify(sc, belief, plan.astype(np.float64), 0, 0, prec=32)
    assert np.array_equal(th, oth)
    agree = np.mean(ft == oft)
    print(f"verification per-sample failure-time agreement {agree:.4f}, fails gpu {fc.sum()} oracle {ofc.sum()}")
    assert agree >= 0.98
    assert abs(int(fc.sum()) - int(ofc.sum())) <= max(5, 0.02 * ofc.sum())


def test_full_steps_match_oracle(gpu):
    """Three closed-loop-style control steps through dr_mppi_step against the oracle
    composition of the same steps (warm-start shift, temperature adaptation, plan
    verification and selection included)."""
    sc = small_mppi(True, K=1024, T=40, n_verif=2048, noise=True)
    rng = np.random.default_rng(5)
    nominal = random_nominal(sc, rng, 0.3)
    ctl = mppi_ctl(sc, nominal=nominal, exact_verify=True)
    ctl.engine = object()
    ref = OracleMPPI(sc, nominal=nominal)
    belief = sc.belief()
    for k in range(3):
        a = ctl.getControl(sc.state)
        oa, info = ref.get_control(sc.state, belief)
        np.testing.assert_allclose(a, oa, rtol=2e-3, atol=2e-3)
        assert ctl.useNewPlan == info["use_new"]
        np.testing.assert_allclose(ctl.h_nominal.reshape(ref.h_nominal.shape), ref.h_nominal, rtol=2e-3, atol=2e-3)
        assert abs(ctl.invTemperature - ref.lam) <= 1e-6 * ref.lam


def test_batch_equals_single(gpu):
    scs = [S.circle_race(agent=a, K=512, T=32, n_verif=512) for a in range(3)]
    singles = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    batched = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    batch = drb.controllers.MPPIBatch(batched)
    for c in singles:
        c.engine = object()
    beliefs = np.stack([s.belief() for s in scs])
    for k in range(2):
        a1 = np.stack([c.getControl(s.state) for c, s in zip(singles, scs)])
        a2 = batch.step([s.state for s in scs], beliefs)
        assert np.array_equal(a1, a2)
        for c1, c2 in zip(singles, batched):
            assert np.array_equal(c1.h_nominal, c2.h_nominal)


def test_graph_replay_equals_eager(gpu):
    scs = [S.circle_race(agent=a, K=256, T=32, n_verif=256) for a in range(2)]
    A = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    Bc = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(Bc)
    bb.set_graph(False)
    bb.set_overlap(False)  # eager, in-order reference for the graph-replayed, overlapped batch
    beliefs = np.stack([s.belief() for s in scs])
    for k in range(4):
        x = ba.step([s.state for s in scs], beliefs)
        y = bb.step([s.state for s in scs], beliefs)
        assert np.array_equal(x, y)
