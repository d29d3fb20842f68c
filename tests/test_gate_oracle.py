"""Gate race (the reference's EnvDroneRace): the oracle port against golden outputs of the
reference built with USE_ENV_DRONERACE, against that build live where present, and its
FP32 error against the FP64 transcription."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import O, drb
from helpers import small_gate, toward_opponent_plan

GOLD = Path(__file__).resolve().parent / "golden"
S = drb.scenarios


@pytest.mark.parametrize("variant,spl", [("gate_spline", True), ("gate_dense", False)])
def test_gate_oracle_matches_reference_golden(variant, spl):
    g = np.load(GOLD / f"{variant}.npz")
    sc = small_gate(spl, K=64, T=40, n_verif=256, seed=int(g["seed"]), noise=True, agent=1, gap=0.02)
    step = int(g["step"])
    noise = O.mppi_noise(sc, step)
    assert np.array_equal(noise, g["noise"])
    B = O.spline_matrix(sc.mppi) if spl else None
    ct, bu, bt = O.mppi_rollout(sc, g["belief"], g["knots_in"], noise, B, step, prec=32)
    assert np.array_equal(ct, g["costs_true"])
    assert np.array_equal(bu, g["branch_used"]) and np.array_equal(bt, g["branch_time"])
    kn, dense, mins, nu, costs = O.mppi_update(sc, g["belief"], ct, bu, bt, noise, B, g["knots_in"], prec=32)
    assert np.array_equal(kn.astype(np.float32), g["knots_out"])
    assert np.array_equal(dense.astype(np.float32), g["dense"])
    assert np.array_equal(mins.astype(np.float32), g["min_costs"])
    assert np.array_equal(nu.astype(np.float32), g["nu"])
    assert np.array_equal(costs.astype(np.float32), g["costs"])
    fc, ft, _ = O.mppi_verify(sc, g["belief"], g["plan"].astype(np.float64), step, 0, prec=32)
    assert fc.sum() > 0
    assert np.array_equal(fc, g["fail_count"]) and np.array_equal(ft, g["fail_time"])


def test_gate_fp32_against_fp64_transcription():
    g = np.load(GOLD / "gate_dense.npz")
    sc = small_gate(False, K=64, T=40, n_verif=256, seed=int(g["seed"]), noise=True, agent=1, gap=0.02)
    ct32, _, _ = O.mppi_rollout(sc, g["belief"], g["knots_in"], g["noise"], None, int(g["step"]), prec=32)
    ct64, _, _ = O.mppi_rollout(sc, g["belief"], g["knots_in"], g["noise"], None, int(g["step"]), prec=64)
    rel = np.abs(ct32 - ct64) / np.maximum(1.0, np.abs(ct64))
    print(f"gate rollout cost FP32 vs FP64: median rel {np.median(rel):.2e}, 99th pct {np.percentile(rel, 99):.2e}")
    assert np.median(rel) < 1e-5


def test_gate_scenario_runs_a_lap_without_terminal_events():
    """The benchmark's gate workload: 64 steps of coasting from each agent's start end in
    no collision, no win and no lap (so every rollout step does full work)."""
    for agent in range(4):
        sc = S.gate_race(agent=agent, K=64, T=64, n_verif=64)
        st, bel = sc.state, sc.belief()
        for t in range(64):
            term, st, bel = O.gate_env_step(sc, 0, np.zeros(2, np.float32), st, bel, apply_noise=False, t=t)
            assert term == 0
        assert list(st.laps) == [0, 0]


@pytest.mark.skipif(not O.ref_available("gate_dense"), reason="reference build not present")
@pytest.mark.parametrize("spl", [True, False])
def test_gate_port_equals_reference_host_code_live(spl):
    """Larger random cases, port vs the reference's gate-race model functions compiled
    here: rollouts with PID action noise (Philox on both sides), the update, a failing
    verification, single environment steps with noise and the costs."""
    variant = O.gate_variant_name(spl)
    sc = small_gate(spl, K=256, T=40, n_verif=512, seed=99, noise=True, agent=2)
    rng = np.random.default_rng(7)
    M = O.mk(sc.mppi)
    knots = rng.normal(0, 1.5, (3, M, 2)).astype(np.float32)
    noise = O.mppi_noise(sc, 5)
    B = O.spline_matrix(sc.mppi) if spl else None
    belief = np.array([0.7, 0.3], np.float32)
    a = O.mppi_rollout(sc, belief, knots, noise, B, 5, prec=32)
    b = O.mppi_rollout(sc, belief, knots, noise, B, 5, impl=variant, nthreads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    ua = O.mppi_update(sc, belief, a[0], a[1], a[2], noise, B, knots, prec=32)
    ub = O.mppi_update(sc, belief, a[0], a[1], a[2], noise, B, knots, impl=variant, nthreads=4)
    for x, y in zip(ua, ub):
        assert np.array_equal(np.asarray(x, np.float32), np.asarray(y, np.float32))
    sc2 = small_gate(spl, K=64, T=40, n_verif=512, seed=5, noise=True, agent=3, gap=0.02)
    plan = toward_opponent_plan(sc2)
    fa, ta, _ = O.mppi_verify(sc2, sc2.belief(), plan.astype(np.float64), 1, 1, prec=32)
    fb, tb, _ = O.mppi_verify(sc2, sc2.belief(), plan, 1, 1, impl=variant, nthreads=4)
    assert fa.sum() > 0 and np.array_equal(fa, fb) and np.array_equal(ta, tb)
    st, bel = sc.state, sc.belief()
    for t in range(30):
        act = rng.normal(0, 3, 2).astype(np.float32)
        ra = O.gate_env_step(sc, 1, act, st, bel, step=t, t=t)
        rb = O.gate_env_step(sc, 1, act, st, bel, step=t, t=t, impl=variant)
        assert ra[0] == rb[0]
        assert bytes(ra[1]) == bytes(rb[1]) and np.array_equal(ra[2], rb[2])
        assert np.array_equal(O.gate_costs(sc, ra[1]), O.gate_costs(sc, ra[1], impl=variant))
        st, bel = ra[1], ra[2]
