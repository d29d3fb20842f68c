"""The algorithmic FLOPs per environment step that bench.py divides by (its roofline
fractions) are what the oracle's operation counter gives for the benchmark workloads
(oracle/count_flops.py: the searches of the track projection counted as the kernels run
them, work whose result nothing reads left out), so the constants cannot drift from the
code. CPU only."""
from __future__ import annotations

import importlib.util

import numpy as np

from conftest import ROOT, O, drb


def _module(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_flop_constants_match_the_oracle_counts():
    cf = _module("count_flops", ROOT / "oracle" / "count_flops.py")
    bench = _module("bench_for_counts", ROOT / "bench.py")
    S, P = drb.scenarios, O.port()
    skip, local = 4, 8
    strat = S.circle_race(agent=0, seed=0, K=4096, T=64, use_splines=False, n_theta=2, n_verif=2**17)
    gate = S.gate_race(agent=0, seed=0, K=4096, T=64, use_splines=False, n_verif=2**17, n_gates=bench.N_GATES)
    pr = S.robust_race(agent=0, seed=0, K=bench.K_PR, T=64, P=bench.P_PR, n_theta=bench.NTH_PR)
    got = {
        "FLOPS_PER_ROLLOUT_STEP": cf._count(P.orc_count_ops, strat, 0, 1 | skip | local),
        "FLOPS_PER_VERIFY_STEP": cf._count(P.orc_count_ops, strat, 1, 2 | skip | local),
        "GATE_FLOPS_PER_ROLLOUT_STEP": cf._count(P.orc_gate_count_ops, gate, 0, 1 | skip | local),
        "GATE_FLOPS_PER_VERIFY_STEP": cf._count(P.orc_gate_count_ops, gate, 1, 2 | skip | local),
        "PR_FLOPS_PER_ROLLOUT_STEP": cf._count_pr(P, pr, 1 | local),
    }
    for name, value in got.items():
        assert np.isclose(getattr(bench, name), value, atol=0.051), (name, getattr(bench, name), value)
    # the searches as the kernels run them do less work than the scans as written
    assert got["FLOPS_PER_VERIFY_STEP"] < cf._count(P.orc_count_ops, strat, 1, 2 | skip)
    assert got["GATE_FLOPS_PER_VERIFY_STEP"] < cf._count(P.orc_gate_count_ops, gate, 1, 2 | skip)
