"""Generates the golden fixtures in this directory from the reference itself.

  * tracks.npz     track grids of the reference's Python front-end (python-src/utils.py:
                   StratRaceEnvironmentConfig.__post_init__, imported from the reference
                   sources) for its round track (python-src/main.py:867-868).
  * wire_*.bin     configuration headers packed by the reference's BytePacker
                   (python-src/protocol.py:13-72) for the stratRaceEnv presets and its
                   tinyGateEnv (wire_gate_mppi.bin).
  * mppi_*.npz     rollout / update / verification outputs of the reference's own model
                   functions compiled from its sources (oracle/_ref, host build) on small
                   cases with perturbations from the Philox streams.
  * pr_*.npz       the same for PR-MPPI.
  * gate_*.npz     the same for the gate race (the reference built with USE_ENV_DRONERACE).
  * cp.npz         Clopper-Pearson bounds from scipy.stats.beta.ppf.

Run from the repository root, with the reference checkout in $DR_REFERENCE (default: a
directory named reference beside the repository):
    python tests/golden/gen_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))

from conftest import O, drb  # noqa: E402

REF = O.reference_dir()

S = drb.scenarios
abi = drb.abi


def ref_python():
    """The reference's python-src modules, with a stand-in for its matplotlib renderer."""
    sys.modules.setdefault("renderer", types.SimpleNamespace(EnvironmentRenderer=object))
    sys.path.insert(0, str(REF / "python-src"))
    import protocol  # noqa: F401
    import utils

    return utils, protocol


def gen_tracks(utils):
    def roundTrack(f):
        return 6 * np.array([np.cos(2 * np.pi * f), np.sin(2 * np.pi * f)])

    oc = utils.StratRaceEnvironmentConfig.OppConfig.preset(droneRadius=0.4, nOpps=1, s1="insensitive", s3="default")
    e = utils.StratRaceEnvironmentConfig(nModelFactors=1, modelSizes=np.array([1]), nOppAgents=1, dt=0.1, droneRadius=0.4, maxSpeed=np.array([3, 2]),
                                         maxAccel=np.array([2, 3]), trackWidth=2, opponentConfigs=(oc,), kV=5, maxOppLatDistFact=1.9,
                                         trackFunction=roundTrack)
    np.savez_compressed(HERE / "tracks.npz", track_length=np.float64(e.trackLength), p_grid=e.p_grid, dp_grid=e.dp_grid, t_grid=e.t_grid,
                        kappa_grid=e.kappa_grid)


def gen_wire(utils, protocol):
    """MSG_HEADER frames as ZMQRecv.runSim sends them (protocol.py:225-229)."""
    sys.path.insert(0, str(REF / "python-src"))
    import main as ref_main

    for name, kw in [("mppi_spline", dict(usePR=False, useSplines=True)), ("mppi_dense", dict(usePR=False, useSplines=False)),
                     ("prmppi", dict(usePR=True, useSplines=True))]:
        env, init, cont, _ = ref_main.stratRaceEnv(mppiPos=0, nConfigs=2, firstConfig=0, **kw)
        frames = []
        for obj in (env, cont, init):
            p = protocol.BytePacker()
            p.pushInt(utils.MSG_TYPE.MSG_HEADER)
            p.pushObj(obj)
            frames.append(p.toBytes())
        with open(HERE / f"wire_{name}.bin", "wb") as f:
            for fr in frames:
                f.write(len(fr).to_bytes(4, "little"))
                f.write(fr)


def gen_wire_gate(utils, protocol):
    """The same frames for the reference's tinyGateEnv (python-src/main.py:40-220, one
    round obstacle, spline MPPI)."""
    sys.path.insert(0, str(REF / "python-src"))
    import main as ref_main

    env, init, cont, _ = ref_main.tinyGateEnv(roundObs=True, useSplines=True, usePR=False)
    frames = []
    for obj in (env, cont, init):
        p = protocol.BytePacker()
        p.pushInt(utils.MSG_TYPE.MSG_HEADER)
        p.pushObj(obj)
        frames.append(p.toBytes())
    with open(HERE / "wire_gate_mppi.bin", "wb") as f:
        for fr in frames:
            f.write(len(fr).to_bytes(4, "little"))
            f.write(fr)


def gen_mppi(variant: str, spl: bool):
    from helpers import small_mppi

    sc = small_mppi(spl, K=64, T=24, M=8, n_verif=256, seed=11, noise=True)
    rng = np.random.default_rng(5)
    c = sc.mppi
    nbp, M = sc.n_theta + 1, O.mk(c)
    knots = rng.normal(0, 0.7, (nbp, M, 2)).astype(np.float32)
    belief = np.array([0.45, 0.55], np.float32)
    noise = O.mppi_noise(sc, 3)
    B = O.spline_matrix(c) if spl else None
    Bref = np.zeros_like(B) if spl else None
    if spl:
        assert O.ref(variant).refh_spline_matrix(C.byref(sc.env), C.byref(c), O._f(Bref)) == 0
        assert np.array_equal(B, Bref)
    ct, bu, bt = O.mppi_rollout(sc, belief, knots, noise, B, 3, impl=variant, nthreads=4)
    kn, dense, mins, nu, costs = O.mppi_update(sc, belief, ct, bu, bt, noise, B, knots, impl=variant, nthreads=4)
    plan = rng.normal(0, 1.0, (nbp, c.n_timesteps, 2)).astype(np.float32)
    fc, ft, _ = O.mppi_verify(sc, belief, plan, 3, 1, impl=variant, nthreads=4)
    np.savez_compressed(HERE / f"mppi_{variant}.npz", knots_in=knots, belief=belief, noise=noise, B=B if spl else np.zeros(1, np.float32), step=3,
                        seed=sc.seed, costs_true=ct, branch_used=bu, branch_time=bt, knots_out=kn, dense=dense, min_costs=mins, nu=nu, costs=costs,
                        plan=plan, fail_count=fc, fail_time=ft)


def gen_gate(variant: str, spl: bool):
    """Gate race (the reference built with USE_ENV_DRONERACE): rollout, update and a
    verification whose plan drives the ego into the opponent."""
    from helpers import small_gate, toward_opponent_plan

    sc = small_gate(spl, K=64, T=40, n_verif=256, seed=13, noise=True, agent=1, gap=0.02)
    rng = np.random.default_rng(9)
    c = sc.mppi
    nbp, M = sc.n_theta + 1, O.mk(c)
    knots = rng.normal(0, 1.0, (nbp, M, 2)).astype(np.float32)
    belief = np.array([0.4, 0.6], np.float32)
    noise = O.mppi_noise(sc, 2)
    B = O.spline_matrix(c) if spl else None
    ct, bu, bt = O.mppi_rollout(sc, belief, knots, noise, B, 2, impl=variant, nthreads=4)
    kn, dense, mins, nu, costs = O.mppi_update(sc, belief, ct, bu, bt, noise, B, knots, impl=variant, nthreads=4)
    plan = toward_opponent_plan(sc)
    fc, ft, _ = O.mppi_verify(sc, belief, plan, 2, 0, impl=variant, nthreads=4)
    assert fc.sum() > 0
    np.savez_compressed(HERE / f"{variant}.npz", knots_in=knots, belief=belief, noise=noise, B=B if spl else np.zeros(1, np.float32), step=2,
                        seed=sc.seed, costs_true=ct, branch_used=bu, branch_time=bt, knots_out=kn, dense=dense, min_costs=mins, nu=nu, costs=costs,
                        plan=plan, fail_count=fc, fail_time=ft)


def gen_pr(variant: str, nth: int):
    sc = S.strat_race(use_pr=True, K=64, T=24) if nth == 2 else S.robust_race(agent=1, seed=2, K=64, T=24, P=8, n_theta=nth)
    sc.prmppi = S.make_prmppi(K=64, T=24, P=8, inv_temperature=1.0, sampling_noise=1.0) if nth == 2 else sc.prmppi
    rng = np.random.default_rng(6)
    T = sc.prmppi.n_timesteps
    nom = rng.normal(0, 0.7, (T, 2)).astype(np.float32)
    rob = rng.normal(0, 0.7, (T, 2)).astype(np.float32)
    belief = sc.belief()
    noise = O.pr_noise(sc, 2)
    th = O.pr_thetas(sc, 2, belief)
    cn, cr = O.pr_rollout(sc, nom, rob, noise, th, 2, impl=variant, nthreads=4)
    full, safe = O.pr_candidates(sc, nom, rob, th, 2, O.S_PR_CAND_ENV, impl=variant)
    np.savez_compressed(HERE / f"pr_{variant}.npz", nom=nom, rob=rob, belief=belief, noise=noise, thetas=th, step=2, seed=sc.seed, cost_nom=cn,
                        cost_rob=cr, cand_full=full, cand_safe=safe)


def gen_cp():
    from scipy.stats import beta

    rows = []
    for n in (100, 10000, 131072, 1000000):
        for k in sorted({0, 1, 2, 5, 17, n // 1000, n // 10, n // 2, n - 1, n}):
            for alpha in (1e-6, 5e-6, 1e-5, 0.05):
                lo = 0.0 if k == 0 else beta.ppf(alpha, k, n - k + 1)
                hi = 1.0 if k == n else beta.ppf(1 - alpha, k + 1, n - k)
                rows.append((k, n, alpha, lo, hi))
    a = np.array(rows, dtype=np.float64)
    np.savez_compressed(HERE / "cp.npz", k=a[:, 0].astype(np.int64), n=a[:, 1].astype(np.int64), alpha=a[:, 2], lower=a[:, 3], upper=a[:, 4])


def main():
    if "--gate" in sys.argv:  # the gate-race fixtures alone
        utils, protocol = ref_python()
        gen_wire_gate(utils, protocol)
        gen_gate("gate_spline", True)
        gen_gate("gate_dense", False)
        return
    utils, protocol = ref_python()
    gen_tracks(utils)
    gen_wire(utils, protocol)
    gen_wire_gate(utils, protocol)
    gen_mppi("nth2_spline", True)
    gen_mppi("nth2_dense", False)
    gen_pr("nth2_spline", 2)
    gen_pr("nth8_spline", 8)
    gen_cp()
    gen_gate("gate_spline", True)
    gen_gate("gate_dense", False)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
