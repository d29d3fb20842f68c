"""PR-MPPI parity on the B200 against the reference's CUDA kernels and the oracle port."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
from helpers import zero_env_noise

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios


def small_pr(nth=2, K=512, T=40, P=8, noise=True):
    if nth == 2:
        sc = S.strat_race(use_pr=True, K=K, T=T)
        sc.prmppi = S.make_prmppi(K=K, T=T, P=P)
    else:
        sc = S.robust_race(agent=0, seed=3, K=K, T=T, P=P, n_theta=nth)
    if not noise:
        zero_env_noise(sc)
    return sc


def _noise_thetas(ctl, sc, belief):
    c = sc.prmppi
    n = np.zeros((c.n_timesteps, c.n_samples, 2), np.float32)
    th = np.zeros(c.P, np.int32)
    abi.check(abi.lib().dr_prmppi_debug_noise(ctl.handle, abi.fptr(belief), abi.fptr(n), n.size, abi.iptr(th)), "pr debug_noise")
    return n, th


@pytest.mark.parametrize("nth", [2, 8])
def test_pr_noise_and_thetas_bit_exact(gpu, nth):
    sc = small_pr(nth)
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed)
    belief = sc.belief()
    n, th = _noise_thetas(ctl, sc, belief)
    assert np.array_equal(n, O.pr_noise(sc, 0))
    assert np.array_equal(th, O.pr_thetas(sc, 0, belief))


@pytest.mark.parametrize("nth,K,T", [(2, 512, 40), (8, 512, 40), (8, 2048, 64)])
def test_pr_rollout_matches_reference_kernel(gpu, nth, K, T):
    """PRMPPIfullRolloutKernel (prmppi_kernels.cu:55-130) on the same perturbation and
    hypotheses: running and safety cost of every (nominal/robust, p, sample). The last case
    is the benchmark's PR-MPPI configuration per agent (8 hypotheses, P 8, K 2048, H 64)."""
    variant = O.ref_variant_name(nth, True)
    sc = small_pr(nth, K=K, T=T, noise=False)
    rng = np.random.default_rng(11)
    nominal = rng.normal(0, 0.8, (sc.prmppi.n_timesteps, 2)).astype(np.float32)
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed, nominal=nominal)
    belief = sc.belief()
    noise, th = _noise_thetas(ctl, sc, belief)
    c = sc.prmppi
    cn = np.zeros((c.P, c.n_samples, 2), np.float32)
    cr = np.zeros_like(cn)
    abi.check(abi.lib().dr_prmppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(cn), abi.fptr(cr)), "pr debug_rollout")
    shifted = np.concatenate([nominal[1:], np.zeros((1, 2), np.float32)])
    rcn = np.zeros_like(cn)
    rcr = np.zeros_like(cn)
    rc = O.ref(variant).refc_pr_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(shifted), O._f(shifted), O._f(noise), O._i(th), 9,
                                        O._f(rcn), O._f(rcr))
    assert rc == 0
    for name, a, b in (("nom", cn, rcn), ("rob", cr, rcr)):
        mism = ~((a == b) | (np.isnan(a) & np.isnan(b)))
        if mism.any():
            idx = np.argwhere(mism)
            rel = np.abs(a - b) / np.maximum(1.0, np.abs(b))
            print(f"{name}: {mism.sum()} differ; per p {mism.any(axis=2).sum(axis=1)}; thetas {th}; samples {np.unique(idx[:, 1])[:20]}")
            for p, s, k in idx[:6]:
                print(f"  p={p} s={s} k={k} mine={a[p, s, k]!r} ref={b[p, s, k]!r} rel={rel[p, s, k]:.2e}")
        assert mism.sum() == 0, f"{name}: {mism.sum()} of {a.size} differ"


def test_pr_steps_match_oracle(gpu):
    """Two control steps through dr_prmppi_step against the oracle composition
    (shift, rollout, cost averaging, three weighted averages, candidate choice,
    safety decision)."""
    sc = small_pr(2, K=512, T=40, noise=True)
    c = sc.prmppi
    ctl = drb.controllers.PRMPPIController(sc.env, c, sc.seed)
    ctl.engine = object()
    belief = sc.belief()
    nom = np.zeros((c.n_timesteps, 2))
    rob = np.zeros((c.n_timesteps, 2))
    lam = np.full(3, c.inv_temperature, np.float32)
    for step in range(2):
        a = ctl.getControl(sc.state)
        nom = np.concatenate([nom[1:], np.zeros((1, 2))])
        rob = np.concatenate([rob[1:], np.zeros((1, 2))])
        noise = O.pr_noise(sc, step)
        th = O.pr_thetas(sc, step, belief)
        cn, cr = O.pr_rollout(sc, nom, rob, noise, th, step)
        cn2, cr2, mins, c1, c2, nr, nu = O.pr_update(sc, cn, cr, noise, nom, rob, lam)
        full, _ = O.pr_candidates(sc, c1, c2, th, step, O.S_PR_CAND_ENV)
        _, safe = O.pr_candidates(sc, c1, c2, th, step, O.S_PR_SAFE_ENV)
        P = c.P
        c1c = np.float32(np.sum(full[:P].astype(np.float32), dtype=np.float32)) / np.float32(P)
        c2c = np.float32(np.sum(full[P:].astype(np.float32), dtype=np.float32)) / np.float32(P)
        chosen = 0 if c1c <= c2c else 1
        use_nom = not np.any(safe[chosen * P:(chosen + 1) * P] > 0)
        nom = c1 if chosen == 0 else c2
        rob = nr
        expect = (nom if use_nom else rob)[0]
        assert ctl.useNomPlan == use_nom
        np.testing.assert_allclose(a, expect, rtol=2e-3, atol=2e-3)
        gn, gr = ctl.nominals()
        np.testing.assert_allclose(gn.reshape(-1, 2), nom, rtol=2e-3, atol=2e-3)
        np.testing.assert_allclose(gr.reshape(-1, 2), rob, rtol=2e-3, atol=2e-3)
        for w in range(3):
            if nu[w] > np.float32(c.max_nu) * np.float32(c.n_samples) and lam[w] > np.float32(0.01):
                lam[w] *= np.float32(0.9)
            elif nu[w] < np.float32(c.min_nu) * np.float32(c.n_samples) and lam[w] < np.float32(100):
                lam[w] *= np.float32(1.2)


def test_env_step_matches_reference(gpu):
    sc = S.strat_race(K=64, T=20)
    st = abi.dr_sim_state.from_buffer_copy(sc.state)
    st_ref = abi.dr_sim_state.from_buffer_copy(sc.state)
    b = sc.belief().copy()
    b_ref = b.copy()
    for k in range(20):
        act = np.array([1.5, -0.5], np.float32)
        term = drb.controllers.env_step(sc.env, 0, act, st, b, True, sc.seed, k)
        term_ref = O.ref("nth2_spline").refh_env_step(C.byref(sc.env), 0, O._f(act), C.byref(st_ref), O._f(b_ref), 1, 0, 2.0, 0, 1, sc.seed, k, 0)
        assert term == term_ref
        np.testing.assert_allclose(np.array(st.pos), np.array(st_ref.pos), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(b, b_ref, rtol=1e-4, atol=1e-6)


def _pr_agents(n=3, K=512, T=40, P=8):
    return [S.robust_race(agent=a, seed=2, K=K, T=T, P=P, n_theta=8) for a in range(n)]


def test_pr_batch_equals_single(gpu):
    """dr_prmppi_batch_step (every agent's kernels in one launch each, graph replay after the
    first step) against each controller stepped alone through dr_prmppi_step."""
    scs = _pr_agents()
    singles = [drb.controllers.PRMPPIController(s.env, s.prmppi, s.seed) for s in scs]
    batched = [drb.controllers.PRMPPIController(s.env, s.prmppi, s.seed) for s in scs]
    batch = drb.controllers.PRMPPIBatch(batched)
    for c in singles:
        c.engine = object()
    beliefs = np.stack([s.belief() for s in scs])
    for k in range(3):
        a1 = np.stack([c.getControl(s.state) for c, s in zip(singles, scs)])
        a2 = batch.step([s.state for s in scs], beliefs)
        assert np.array_equal(a1, a2)
        for c1, c2 in zip(singles, batched):
            for x, y in zip(c1.nominals(), c2.nominals()):
                assert np.array_equal(x, y)


@pytest.mark.parametrize("slots", [2, 4])
def test_pr_rollout_slots_bit_identical(gpu, slots):
    """Several hypothesis slots per rollout thread sharing the ego's moves (the benchmark's
    PR workload: the ego draws no noise, P 8): actions and both plans identical to one slot
    per thread, step after step."""
    scs = _pr_agents()
    assert all(s.env.action_noise_level == 0 and s.env.pos_noise_level == 0 and s.env.speed_noise_level == 0 for s in scs)
    beliefs = np.stack([s.belief() for s in scs])
    out = []
    for n in (1, slots):
        ctls = [drb.controllers.PRMPPIController(s.env, s.prmppi, s.seed) for s in scs]
        b = drb.controllers.PRMPPIBatch(ctls)
        b.set_rollout_slots(n)
        acts = [b.step([s.state for s in scs], beliefs) for _ in range(3)]
        out.append((acts, [c.nominals() for c in ctls]))
        b.close()
    (a1, n1), (a2, n2) = out
    for x, y in zip(a1, a2):
        assert np.array_equal(x, y)
    for p, q in zip(n1, n2):
        assert np.array_equal(p[0], q[0]) and np.array_equal(p[1], q[1])


def test_pr_rollout_slots_fall_back_with_ego_noise(gpu):
    """With ego noise the slots cannot share the ego's moves: the batch keeps one slot per
    thread (same results), and an unsupported count is an error."""
    scs = _pr_agents(n=2)
    for s in scs:
        s.env.action_noise_level = 0.1
    beliefs = np.stack([s.belief() for s in scs])
    res = []
    for n in (1, 4):
        ctls = [drb.controllers.PRMPPIController(s.env, s.prmppi, s.seed) for s in scs]
        b = drb.controllers.PRMPPIBatch(ctls)
        b.set_rollout_slots(n)
        res.append([b.step([s.state for s in scs], beliefs) for _ in range(2)])
        if n == 4:
            with pytest.raises(abi.DrError):
                b.set_rollout_slots(3)
        b.close()
    for x, y in zip(*res):
        assert np.array_equal(x, y)
