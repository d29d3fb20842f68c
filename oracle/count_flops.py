"""Algorithmic FP32 work per environment step of the benchmark workloads, counted on the
oracle's model (oracle/port/opcount.cpp): the constants bench.py divides by to report its
roofline fractions. Test and measurement infrastructure, not part of the product.

    python oracle/count_flops.py

Each count runs 256 samples of the benchmark's first agent from its initial state (zero
plan, the controller's perturbations for the rollout, the noise-free plan for the
verification) and counts every add/sub/mul/div/sqrt/exp/log/pow/min/max once per distinct
operation and operands (comparisons are not FLOPs): within a step (rollout), within a step
index over the samples (verification: the samples share the ego's moves); leaving out work
whose result nothing reads (the belief update and the other hypotheses' opponent actions
once a sample has committed to a branch), as the kernels do; and counting the track
projections' searches as the kernels run them where their certificate holds (the local
search of the window, the gate race's walks without the margin scans they skip; the
benchmark's tracks and racelines certify everywhere a drone can be). The PR-MPPI rollout
is counted over 64 samples under each of its hypotheses, averaged.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def _package():
    spec = importlib.util.spec_from_file_location("drone_race_b200", ROOT / "drone-race_b200" / "__init__.py",
                                                  submodule_search_locations=[str(ROOT / "drone-race_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["drone_race_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _count(fn, sc, kind: int, dedup: int, nsamples: int = 256) -> float:
    from oracle import oracle as O

    c = sc.mppi
    nominal = np.zeros((sc.n_theta + 1, c.n_timesteps, 2), np.float32)
    noise = np.ascontiguousarray(O.mppi_noise(sc, 0), np.float32)
    out = (C.c_double * 10)()
    rc = fn(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(sc.belief()), O._f(nominal), O._f(noise), sc.seed, 0, nsamples, kind, dedup, out)
    assert rc == 0
    return sum(out[:8]) / out[9]


def _count_pr(P, sc, dedup: int, nsamples: int = 64) -> float:
    from oracle import oracle as O

    c = sc.prmppi
    nominal = np.zeros((c.n_timesteps, 2), np.float32)
    noise = np.ascontiguousarray(O.pr_noise(sc, 0), np.float32)
    per = []
    for theta in range(sc.env.n_theta):
        out = (C.c_double * 10)()
        rc = P.orc_pr_count_ops(C.byref(sc.env), C.byref(c), C.byref(sc.state), O._f(nominal), O._f(noise), theta, sc.seed, 0, nsamples, dedup, out)
        assert rc == 0
        per.append(sum(out[:8]) / out[9])
    return float(np.mean(per))


def main() -> None:
    drb = _package()
    from oracle import oracle as O

    O.set_abi(drb.abi)
    S = drb.scenarios
    P = O.port()
    strat = S.circle_race(agent=0, seed=0, K=4096, T=64, use_splines=False, n_theta=2, n_verif=2**17)
    gate = S.gate_race(agent=0, seed=0, K=4096, T=64, use_splines=False, n_verif=2**17, n_gates=8)
    skip, local = 4, 8
    print(f"strategic race: rollout {_count(P.orc_count_ops, strat, 0, 1 | skip | local):.1f}, "
          f"verification {_count(P.orc_count_ops, strat, 1, 2 | skip | local):.1f}")
    print(f"gate race:      rollout {_count(P.orc_gate_count_ops, gate, 0, 1 | skip | local):.1f}, "
          f"verification {_count(P.orc_gate_count_ops, gate, 1, 2 | skip | local):.1f}")
    pr = S.robust_race(agent=0, seed=0, K=2048, T=64, P=8, n_theta=8)
    print(f"PR-MPPI rollout: {_count_pr(P, pr, 1 | local):.1f} (window scans as written: {_count_pr(P, pr, 1):.1f})")
    print(f"(window scans as written: strategic {_count(P.orc_count_ops, strat, 0, 1 | skip):.1f} / {_count(P.orc_count_ops, strat, 1, 2 | skip):.1f}, "
          f"gate {_count(P.orc_gate_count_ops, gate, 0, 1 | skip):.1f} / {_count(P.orc_gate_count_ops, gate, 1, 2 | skip):.1f})")
    print(f"(as the reference writes them, no sharing: strategic {_count(P.orc_count_ops, strat, 0, 0):.1f} / {_count(P.orc_count_ops, strat, 1, 0):.1f}, "
          f"gate {_count(P.orc_gate_count_ops, gate, 0, 0):.1f} / {_count(P.orc_gate_count_ops, gate, 1, 0):.1f})")


if __name__ == "__main__":
    main()
