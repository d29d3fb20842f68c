"""The Monte-Carlo verification's fast flavour (the default) against the reference's own
verifyNominalFailureKernel (kernels.cu:488-551, compiled from the reference sources into
oracle/_ref) and against this library's exact flavour, in distribution.

The reference draws each sample's hypothesis and the opponents' action noise from curand,
so its failure counts are reproducible only statistically; the fast flavour draws its own
(Philox, Box-Muller) and evaluates the model with the hardware's approximate division,
square root and exponential. With V samples each, the failure fraction up to step t of two
independent runs differs by less than 5 standard deviations of a difference of binomial
proportions, for every t (a Kolmogorov-Smirnov-style band over the horizon). The case:
the benchmark's strategic race (K and V of the benchmark, V = 2^17, horizon 40) with the ego
1.2 m behind the opponent and a plan that accelerates it at the opponent, so that about
two thirds of the samples collide, at steps 20-35, mostly under the blocking hypothesis.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios

Z = 5.0  # standard deviations allowed between two independent Monte-Carlo estimates


def _case(gap=1.2, noise=0.5, accel=6.0, V=2**17, nopp=1, nth=2):
    sc = S.circle_race(agent=0, seed=0, K=256, T=64, use_splines=False, n_theta=nth, n_verif=V)
    sc.state = S.initial_state(sc.grids, S._start_indices(sc.grids, 3.0, gap, 0), 1)
    for th in range(nth):
        sc.env.opp_configs[th].action_noise[0] = noise
    st = sc.state
    d = np.array([st.pos[2] - st.pos[0], st.pos[3] - st.pos[1]], np.float64)
    d = d / np.linalg.norm(d) * accel
    plan = np.broadcast_to(d, (nth + 1, sc.mppi.n_timesteps, 2)).astype(np.float32).copy()
    return sc, plan


def _ours(sc, plan, exact, ego=True, belief=None):
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed)
    if exact:
        ctl.set_verify_exact(True)
    if not ego:
        ctl.set_ego_table(False)
    T, V = sc.mppi.n_timesteps, sc.mppi.n_verif_samples
    fc = np.zeros(T, np.uint32)
    ft = np.zeros(V, np.int32)
    th = np.zeros(V, np.int32)
    bel = sc.belief() if belief is None else np.asarray(belief, np.float32)
    abi.check(abi.lib().dr_mppi_debug_verify(ctl.handle, C.byref(sc.state), abi.fptr(bel), abi.fptr(plan), 0, abi.uptr(fc), abi.iptr(ft),
                                             abi.iptr(th)), "debug_verify")
    return fc, ft, th


def _reference(sc, plan, seed):
    fc = np.zeros(sc.mppi.n_timesteps, np.uint32)
    rc = O.ref(O.ref_variant_name(sc.n_theta, False)).refc_mppi_verify(C.byref(sc.env), C.byref(sc.mppi), C.byref(sc.state), O._f(sc.belief()),
                                                                      O._f(plan), seed, O._u(fc))
    assert rc == 0
    return fc


def _same_distribution(a, b, V, what):
    """Cumulative failure fractions of two independent runs of V samples each."""
    Fa = np.cumsum(a.astype(np.float64)) / V
    Fb = np.cumsum(b.astype(np.float64)) / V
    p = 0.5 * (Fa + Fb)
    sd = np.sqrt(np.maximum(p * (1 - p), 1.0 / V) * 2.0 / V)
    z = np.abs(Fa - Fb) / sd
    print(f"{what}: failure fraction {Fa[-1]:.4f} vs {Fb[-1]:.4f}, largest |difference| {np.max(np.abs(Fa - Fb)):.2e} = {z.max():.2f} sd "
          f"(at step {int(np.argmax(z))})")
    assert z.max() < Z, f"{what}: cumulative failure fractions differ by {z.max():.2f} sd"


def test_fast_verification_matches_reference_in_distribution(gpu):
    sc, plan = _case()
    V = sc.mppi.n_verif_samples
    fast, ft, th = _ours(sc, plan, exact=False)
    ref = _reference(sc, plan, 17)
    assert 0.3 < fast.sum() / V < 0.95, "the case must fail on a fair share of the samples"
    _same_distribution(fast, ref, V, "fast flavour vs reference kernel")
    # per-sample records agree with the histogram
    assert np.array_equal(np.bincount(ft[ft >= 0], minlength=len(fast)), fast)
    # hypotheses drawn from the belief (0.5 / 0.5)
    frac1 = th.mean()
    assert abs(frac1 - 0.5) < Z * np.sqrt(0.25 / V)


def test_exact_verification_matches_reference_in_distribution(gpu):
    sc, plan = _case()
    V = sc.mppi.n_verif_samples
    exact, _, _ = _ours(sc, plan, exact=True)
    _same_distribution(exact, _reference(sc, plan, 23), V, "exact flavour vs reference kernel")


@pytest.mark.parametrize("gap,noise", [(1.2, 0.5), (2.0, 2.0)])
def test_fast_matches_exact_in_distribution(gpu, gap, noise):
    """The second case fails rarely (a few per cent, late in the horizon): the tail."""
    sc, plan = _case(gap=gap, noise=noise)
    V = sc.mppi.n_verif_samples
    fast, _, _ = _ours(sc, plan, exact=False)
    exact, _, _ = _ours(sc, plan, exact=True)
    assert exact.sum() > 0
    _same_distribution(fast, exact, V, f"fast vs exact (gap {gap}, noise {noise})")


def test_fast_verification_is_deterministic(gpu):
    sc, plan = _case(V=2**15)
    a, fa, _ = _ours(sc, plan, exact=False)
    b, fb, _ = _ours(sc, plan, exact=False)
    assert np.array_equal(a, b) and np.array_equal(fa, fb)


@pytest.mark.parametrize("gap,noise,belief", [(1.2, 0.5, None), (2.0, 2.0, None), (1.2, 0.5, [0.05, 0.95])])
def test_ego_table_changes_no_failure_time(gpu, gap, noise, belief):
    """The fast verification reads the ego before and after each step from the shared ego
    table (the trajectory without branching, and one per branch and branching step) or moves
    the ego in every sample (dr_mppi_set_ego_table off): the per-sample failure times and
    hypotheses are identical. Cases: samples that branch at many steps, and a confident
    initial belief (the branch is taken before the first step)."""
    sc, plan = _case(gap=gap, noise=noise, V=2**15)
    a, fa, ta = _ours(sc, plan, exact=False, ego=True, belief=belief)
    b, fb, tb = _ours(sc, plan, exact=False, ego=False, belief=belief)
    assert a.sum() > 0
    assert np.array_equal(ta, tb)
    assert np.array_equal(fa, fb), f"{np.sum(fa != fb)} of {fa.size} failure times differ"
    assert np.array_equal(a, b)
