"""Gate race on the B200: the CUDA path against the reference's own CUDA kernels built
with USE_ENV_DRONERACE (oracle/_ref) on identical injected perturbations, and against the
CPU oracle port with the in-rollout noise on."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
from helpers import OracleMPPI, random_nominal, small_gate, toward_opponent_plan

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios


def _ctl(sc, nominal=None, exact_verify=False):
    """exact_verify: the verification's exact flavour, whose per-sample results equal the
    oracle's (the tests that compare failure times or plan choices with the oracle)."""
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed, nominal=nominal)
    if exact_verify:
        ctl.set_verify_exact(True)
    return ctl


def _dev_rollout(ctl, sc, belief):
    K, nth = sc.mppi.n_samples, sc.n_theta
    ct = np.zeros((nth, K), np.float32)
    bu = np.zeros((nth, K), np.int32)
    bt = np.zeros((nth, K), np.int32)
    costs = np.zeros((nth + 1, K), np.float32)
    abi.check(abi.lib().dr_gate_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(ct), abi.iptr(bu), abi.iptr(bt),
                                                   abi.fptr(costs)), "debug_rollout")
    return ct, bu, bt, costs


def _dev_noise(ctl, sc):
    c = sc.mppi
    n = np.zeros((sc.n_theta + 1, O.mk(c), c.n_samples, 2), np.float32)
    abi.check(abi.lib().dr_mppi_debug_noise(ctl.handle, abi.fptr(n), n.size), "debug_noise")
    return n


@pytest.mark.parametrize("spl", [True, False])
def test_gate_rollout_matches_reference_kernel(gpu, spl):
    """fullRolloutKernel of the reference built for the gate race vs the fused gate
    rollout, same perturbation, PID noise off: per-sample costs and branch bookkeeping
    identical, and the branch aggregation identical to the reference's update path."""
    variant = O.gate_variant_name(spl)
    sc = small_gate(spl, K=1024, T=40, noise=False, agent=1)
    rng = np.random.default_rng(1)
    ctl = _ctl(sc, nominal=random_nominal(sc, rng, 1.5))
    belief = sc.belief()
    if spl:
        ctl.engine = object()
        ctl.getControl(sc.state)  # a full step first, so that the knots are not all zero
    assert np.array_equal(_dev_noise(ctl, sc), O.mppi_noise(sc, int(abi.lib().dr_mppi_get_step(ctl.handle))))
    noise = _dev_noise(ctl, sc)
    ct, bu, bt, costs = _dev_rollout(ctl, sc, belief)
    kn = ctl.knots()
    assert np.abs(kn).max() > 0
    rct, rbu, rbt = np.zeros_like(ct), np.zeros_like(bu), np.zeros_like(bt)
    B = O.spline_matrix(sc.mppi) if spl else np.zeros(1, np.float32)
    rc = O.ref(variant).refc_mppi_rollout(C.byref(sc.env), C.byref(sc.mppi), C.byref(sc.state), O._f(belief), O._f(np.ascontiguousarray(kn)),
                                          O._f(noise), O._f(B), 123, O._f(rct), O._i(rbu), O._i(rbt))
    assert rc == 0
    assert np.array_equal(bu, rbu) and np.array_equal(bt, rbt)
    mism = ~((ct == rct) | (np.isnan(ct) & np.isnan(rct)))
    assert mism.sum() == 0, f"{mism.sum()} of {ct.size} costs differ; first {np.argwhere(mism)[:5]}"
    rcosts = np.zeros_like(costs)
    dummy = np.zeros((sc.n_theta + 1) * sc.mppi.n_timesteps * 2, np.float32)
    mins = np.zeros((sc.n_theta + 1) * O.mk(sc.mppi), np.float32)
    nu = np.zeros(sc.n_theta + 1, np.float32)
    rc = O.ref(variant).refc_mppi_update(C.byref(sc.env), C.byref(sc.mppi), O._f(belief), O._f(rct), O._i(rbu), O._i(rbt), O._f(noise), O._f(B),
                                         O._f(np.ascontiguousarray(kn).copy()), O._f(dummy), O._f(mins), O._f(nu), O._f(rcosts))
    assert rc == 0
    assert np.array_equal(costs, rcosts)


@pytest.mark.parametrize("spl", [True, False])
def test_gate_update_matches_reference_kernels(gpu, spl):
    """The shared update kernels on gate-race rollout outputs against the reference's
    update kernels built for the gate race (the clamp uses the ego's maxAccel[iMppi])."""
    variant = O.gate_variant_name(spl)
    sc = small_gate(spl, K=1024, T=40, noise=False, agent=2)
    rng = np.random.default_rng(2)
    ctl = _ctl(sc, nominal=random_nominal(sc, rng, 2.0))
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
    r_kn, r_dense, r_mins, r_nu = kn.copy(), np.zeros_like(dense), np.zeros_like(mins), np.zeros_like(nu)
    rc = O.ref(variant).refc_mppi_update(C.byref(sc.env), C.byref(sc.mppi), O._f(belief), O._f(ct32), O._i(bu), O._i(bt), O._f(noise), O._f(B),
                                         O._f(r_kn), O._f(r_dense), O._f(r_mins), O._f(r_nu), None)
    assert rc == 0
    assert np.array_equal(mins, r_mins)
    np.testing.assert_allclose(nu, r_nu, rtol=1e-6)
    np.testing.assert_allclose(new_kn, r_kn, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(dense, r_dense, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("spl", [True, False])
def test_gate_rollout_matches_oracle_with_noise(gpu, spl):
    """PID action noise on (Philox on both sides): the GPU rollout against the FP32 oracle
    port; disagreements only where host and device round differently (FMA contraction)."""
    sc = small_gate(spl, K=1024, T=40, noise=True, agent=0)
    rng = np.random.default_rng(3)
    ctl = _ctl(sc, nominal=random_nominal(sc, rng, 1.5))
    belief = sc.belief()
    kn = ctl.knots().copy()
    B = O.spline_matrix(sc.mppi) if spl else None
    noise = O.mppi_noise(sc, 0)
    ct, bu, bt, _ = _dev_rollout(ctl, sc, belief)
    oct32, obu, obt = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=32)
    oct64, _, _ = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=64)
    rel = np.abs(ct - oct32) / np.maximum(1.0, np.abs(oct32))
    frac = np.mean(rel <= 1e-5)
    rel64 = np.abs(ct - oct64) / np.maximum(1.0, np.abs(oct64))
    print(f"gate: fp32 oracle agreement {frac:.4f}; median |gpu-fp64|/|fp64| {np.median(rel64):.2e}")
    assert frac >= 0.97
    assert np.mean(bu == obu) >= 0.97


def test_gate_verification_matches_oracle(gpu):
    sc = small_gate(False, K=256, T=40, n_verif=4096, noise=True, agent=1, gap=0.02)
    ctl = _ctl(sc, exact_verify=True)
    plan = toward_opponent_plan(sc)
    belief = sc.belief()
    fc = np.zeros(sc.mppi.n_timesteps, np.uint32)
    ft = np.zeros(sc.mppi.n_verif_samples, np.int32)
    th = np.zeros(sc.mppi.n_verif_samples, np.int32)
    abi.check(abi.lib().dr_gate_mppi_debug_verify(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(plan), 0, abi.uptr(fc), abi.iptr(ft),
                                                  abi.iptr(th)), "debug_verify")
    ofc, oft, oth = O.mppi_verify(sc, belief, plan.astype(np.float64), 0, 0, prec=32)
    assert np.array_equal(th, oth)
    agree = np.mean(ft == oft)
    print(f"gate verification per-sample agreement {agree:.4f}, fails gpu {fc.sum()} oracle {ofc.sum()}")
    assert ofc.sum() > 0
    assert agree >= 0.98
    assert abs(int(fc.sum()) - int(ofc.sum())) <= max(5, 0.02 * ofc.sum())


def test_gate_full_steps_match_oracle(gpu):
    """Three control steps through dr_gate_mppi_step against the oracle composition of the
    same steps (shift, temperature, verification of both plans, plan choice)."""
    sc = small_gate(True, K=1024, T=40, n_verif=2048, noise=True, agent=3)
    rng = np.random.default_rng(5)
    nominal = random_nominal(sc, rng, 0.5)
    ctl = _ctl(sc, nominal=nominal, exact_verify=True)
    ctl.engine = object()
    ref = OracleMPPI(sc, nominal=nominal)
    belief = sc.belief()
    for k in range(3):
        a = ctl.getControl(sc.state)
        oa, info = ref.get_control(sc.state, belief)
        np.testing.assert_allclose(a, oa, rtol=2e-3, atol=2e-3)
        assert ctl.useNewPlan == info["use_new"]
        np.testing.assert_allclose(ctl.h_nominal.reshape(ref.h_nominal.shape), ref.h_nominal, rtol=2e-3, atol=2e-3)


def test_gate_batch_equals_single_and_graph_replay(gpu):
    scs = [S.gate_race(agent=a, K=512, T=32, n_verif=512) for a in range(3)]
    singles = [_ctl(s) for s in scs]
    batched = [_ctl(s) for s in scs]
    batch = drb.controllers.MPPIBatch(batched)  # graph replay after the first step, overlap on
    for c in singles:
        c.engine = object()
    beliefs = np.stack([s.belief() for s in scs])
    for k in range(3):
        a1 = np.stack([c.getControl(s.state) for c, s in zip(singles, scs)])
        a2 = batch.step([s.state for s in scs], beliefs)
        assert np.array_equal(a1, a2)
        for c1, c2 in zip(singles, batched):
            assert np.array_equal(c1.h_nominal, c2.h_nominal)


def test_gate_env_step_matches_oracle(gpu):
    sc = small_gate(False, K=64, T=40, noise=True, agent=0)
    st, bel = sc.state, sc.belief()
    rng = np.random.default_rng(8)
    for t in range(20):
        act = rng.normal(0, 3, 2).astype(np.float32)
        term, st_d, bel_d = drb.controllers.gate_env_step(sc.env, 1, act, st, bel, True, sc.seed, t)
        oterm, st_o, bel_o = O.gate_env_step(sc, 1, act, st, bel, step=t, t=0)
        assert term == oterm
        np.testing.assert_allclose(np.array(st_d.pos), np.array(st_o.pos), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(np.array(st_d.vel), np.array(st_o.vel), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(bel_d, bel_o, rtol=1e-4, atol=1e-6)
        assert list(st_d.gates) == list(st_o.gates) and list(st_d.laps) == list(st_o.laps)
        st, bel = st_o, bel_o


def test_gate_state_type_is_checked(gpu):
    sc = small_gate(False, K=64, T=16, noise=False)
    ctl = _ctl(sc)
    out = np.zeros(2, np.float32)
    rc = abi.lib().dr_mppi_step(ctl.handle, C.byref(abi.dr_sim_state()), abi.fptr(sc.belief()), abi.fptr(out), None)
    assert rc == abi.DR_ERR_INVALID_ARG


@pytest.mark.skipif(not (O.REF_DIR / "libadapter_gate.so").exists(), reason="gate adapter build not present")
def test_cpp_adapter_on_the_gate_race(gpu):
    """The C++ drop-in (adapter/controllers.h + controllers_drmppi.cpp) compiled against the
    reference's headers for the gate race: its MPPIController::getControl sequence equals
    the Python controller's on the same configuration (both run this library)."""
    import ctypes as CT

    sc = small_gate(True, K=512, T=32, n_verif=512, noise=True, agent=1)
    L = CT.CDLL(str(O.REF_DIR / "libadapter_gate.so"))
    L.adapter_gate_run.restype = CT.c_int
    L.adapter_gate_run.argtypes = [CT.POINTER(abi.dr_gate_env_config), CT.POINTER(abi.dr_mppi_config), CT.c_int, CT.POINTER(abi.dr_gate_state), CT.c_int,
                                   CT.POINTER(CT.c_float), CT.POINTER(CT.c_float)]
    n, nn = 3, (sc.n_theta + 1) * sc.mppi.n_timesteps * 2
    acts = np.zeros((n, 2), np.float32)
    noms = np.zeros((n, nn), np.float32)
    assert L.adapter_gate_run(CT.byref(sc.env), CT.byref(sc.mppi), sc.seed, CT.byref(sc.state), n, abi.fptr(acts), abi.fptr(noms)) == 0
    ctl = _ctl(sc)
    ctl.engine = object()
    for k in range(n):
        a = ctl.getControl(sc.state)
        assert np.array_equal(a, acts[k])
        assert np.array_equal(ctl.h_nominal, noms[k])



def _gate_fail_counts(sc, plan, exact, seed_ref=None):
    if seed_ref is not None:
        fc = np.zeros(sc.mppi.n_timesteps, np.uint32)
        rc = O.ref(O.gate_variant_name(False)).refc_mppi_verify(C.byref(sc.env), C.byref(sc.mppi), C.byref(sc.state), O._f(sc.belief()),
                                                               O._f(plan), seed_ref, O._u(fc))
        assert rc == 0
        return fc
    ctl = _ctl(sc, exact_verify=exact)
    fc = np.zeros(sc.mppi.n_timesteps, np.uint32)
    abi.check(abi.lib().dr_gate_mppi_debug_verify(ctl.handle, C.byref(sc.state), abi.fptr(sc.belief()), abi.fptr(plan), 0, abi.uptr(fc), None, None),
              "debug_verify")
    return fc


def test_gate_fast_verification_matches_reference_in_distribution(gpu):
    """The gate race's verification in the fast flavour (the default: the hardware's
    approximate division, square root and exponential, Box-Muller PID noise) against the
    reference's verifyNominalFailureKernel built for the gate race (curand hypotheses and
    noise) and against this library's exact flavour: with V = 2^17 samples each, the
    cumulative failure fractions differ by less than 5 standard deviations of a
    difference of two binomial proportions at every step. The case: the ego driven at the
    PID opponent (noise 0.5) from 2 % of a lap behind, so that a fair share collides."""
    sc = small_gate(False, K=256, T=40, n_verif=2**17, noise=True, agent=1, gap=0.02)
    plan = toward_opponent_plan(sc)
    V = sc.mppi.n_verif_samples
    fast = _gate_fail_counts(sc, plan, exact=False)
    exact = _gate_fail_counts(sc, plan, exact=True)
    ref = _gate_fail_counts(sc, plan, exact=False, seed_ref=31)
    assert 0.05 < fast.sum() / V < 0.95, f"failure fraction {fast.sum() / V}"
    for name, a, b in (("fast vs reference", fast, ref), ("fast vs exact", fast, exact), ("exact vs reference", exact, ref)):
        Fa = np.cumsum(a.astype(np.float64)) / V
        Fb = np.cumsum(b.astype(np.float64)) / V
        p = 0.5 * (Fa + Fb)
        sd = np.sqrt(np.maximum(p * (1 - p), 1.0 / V) * 2.0 / V)
        z = np.abs(Fa - Fb) / sd
        print(f"{name}: failure fraction {Fa[-1]:.4f} vs {Fb[-1]:.4f}, largest difference {z.max():.2f} sd")
        assert z.max() < 5.0, f"{name}: {z.max():.2f} sd"
