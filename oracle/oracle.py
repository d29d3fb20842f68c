"""TEST INFRASTRUCTURE (oracle). Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module, and only as the checker.

ctypes wrappers for
  * the oracle port (oracle/_build/liborc_port.so, built from oracle/port/): the
    CPU restatement of the reference's MPPI / PR-MPPI path in FP32 and FP64;
  * the reference itself (oracle/_ref/libref_<variant>.so, built from the reference
    sources by oracle/Makefile): host loops over its model functions (refh_*) and
    launches of its CUDA kernels (refc_*, GPU box only).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
PORT_LIB = ORACLE_DIR / "_build" / "liborc_port.so"
REF_DIR = ORACLE_DIR / "_ref"

_abi = None


def set_abi(abi_module) -> None:
    """The oracle takes the boundary types (dr_env_config, ...) from the package's abi module."""
    global _abi
    _abi = abi_module


def _types():
    assert _abi is not None, "call oracle.set_abi(abi) first"
    return _abi


def reference_dir() -> Path:
    """The reference checkout: $DR_REFERENCE, else a directory named `reference` beside
    the repository (the layout oracle/Makefile assumes too)."""
    env = os.environ.get("DR_REFERENCE")
    return Path(env) if env else ORACLE_DIR.parents[1] / "reference"


def build(ref: bool = True) -> None:
    """Compile the oracle (make -C oracle). The reference variants need the reference
    sources, present only where the oracle is built (not on the GPU box, which uses the
    prebuilt libraries)."""
    import subprocess

    targets = ["port"]
    if ref and reference_dir().exists():
        targets += ["ref", "engine", "adapter_gate"]
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "-j4", *targets], check=True)


_port = None


def port() -> C.CDLL:
    global _port
    if _port is None:
        a = _types()
        L = C.CDLL(str(PORT_LIB))
        P = C.POINTER
        f, d, i, u = P(C.c_float), P(C.c_double), P(C.c_int32), P(C.c_uint32)
        E, M, PR, S = P(a.dr_env_config), P(a.dr_mppi_config), P(a.dr_prmppi_config), P(a.dr_sim_state)
        GE, GS = P(a.dr_gate_env_config), P(a.dr_gate_state)
        u64 = C.c_uint64
        protos = {
            "orc_mppi_noise": (None, [u64, u64, C.c_int, C.c_int, C.c_int, f, f]),
            "orc_pr_noise": (None, [u64, u64, C.c_int, C.c_int, f, f]),
            "orc_pr_thetas": (None, [u64, u64, C.c_int, C.c_int, f, i]),
            "orc_philox": (None, [C.c_uint32] * 6 + [u]),
            "orc_normals_from_words": (None, [u, C.c_int, f]),
            "orc_series_logf": (C.c_float, [C.c_float]),
            "orc_mppi_rollout": (C.c_int, [C.c_int, E, M, S, f, f, f, f, u64, u64, d, i, i]),
            "orc_mppi_update": (C.c_int, [C.c_int, E, M, f, d, i, i, f, f, d, d, d, d, d, C.c_int]),
            "orc_mppi_verify": (C.c_int, [C.c_int, E, M, S, f, d, u64, u64, C.c_int, u, i, i]),
            "orc_spline_matrix": (None, [C.c_int, C.c_int, i, f]),
            "orc_shift_spline": (None, [M, f, d, C.c_int, C.c_int]),
            "orc_cp_lower": (C.c_double, [C.c_uint, C.c_uint, C.c_double]),
            "orc_cp_upper": (C.c_double, [C.c_uint, C.c_uint, C.c_double]),
            "orc_pr_rollout": (C.c_int, [C.c_int, E, PR, S, d, d, f, i, u64, u64, d, d]),
            "orc_pr_update": (C.c_int, [C.c_int, PR, d, d, f, d, d, f, d, d, d, d, d, C.c_int]),
            "orc_pr_candidates": (C.c_int, [C.c_int, E, PR, S, d, d, i, u64, u64, C.c_int, d, d]),
            "orc_env_step": (C.c_int, [C.c_int, E, C.c_int, f, S, f, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, u64, u64, C.c_int]),
            "orc_costs": (None, [E, M, PR, S, f]),
            "orc_gate_rollout": (C.c_int, [C.c_int, GE, M, GS, f, f, f, f, u64, u64, d, i, i]),
            "orc_gate_update": (C.c_int, [C.c_int, GE, M, f, d, i, i, f, f, d, d, d, d, d, C.c_int]),
            "orc_gate_verify": (C.c_int, [C.c_int, GE, M, GS, f, d, u64, u64, C.c_int, u, i, i]),
            "orc_gate_env_step": (C.c_int, [C.c_int, GE, C.c_int, f, GS, f, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int, u64, u64,
                                            C.c_int]),
            "orc_gate_costs": (None, [GE, M, GS, f]),
            "orc_count_ops": (C.c_int, [E, M, S, f, f, f, u64, u64, C.c_int, C.c_int, C.c_int, d]),
            "orc_gate_count_ops": (C.c_int, [GE, M, GS, f, f, f, u64, u64, C.c_int, C.c_int, C.c_int, d]),
            "orc_nominal_cost": (C.c_int, [E, M, S, f, f, d, d, d, d, d, i]),
            "orc_pr_count_ops": (C.c_int, [E, PR, S, f, f, C.c_int, u64, u64, C.c_int, C.c_int, d]),
        }
        for n, (r, args) in protos.items():
            fn = getattr(L, n)
            fn.restype = r
            fn.argtypes = args
        _port = L
    return _port


_refs: dict[str, C.CDLL] = {}


def ref_variant_name(n_theta: int, use_splines: bool) -> str:
    return f"nth{n_theta}_{'spline' if use_splines else 'dense'}"


def gate_variant_name(use_splines: bool) -> str:
    """The reference compiled for the gate race (EnvDroneRace, N_TRUE_MODELS = 2)."""
    return f"gate_{'spline' if use_splines else 'dense'}"


def ref_available(variant: str) -> bool:
    return (REF_DIR / f"libref_{variant}.so").exists()


def ref(variant: str) -> C.CDLL:
    if variant not in _refs:
        a = _types()
        L = C.CDLL(str(REF_DIR / f"libref_{variant}.so"))
        P = C.POINTER
        f, d, i, u = P(C.c_float), P(C.c_double), P(C.c_int32), P(C.c_uint32)
        E, M, PR, S = P(a.dr_env_config), P(a.dr_mppi_config), P(a.dr_prmppi_config), P(a.dr_sim_state)
        if variant.startswith("gate"):  # the same entry points on the gate race's structs
            E, S = P(a.dr_gate_env_config), P(a.dr_gate_state)
        u64, I = C.c_uint64, C.c_int
        protos = {
            "ref_n_theta": (I, []),
            "ref_n_opp": (I, []),
            "ref_use_splines": (I, []),
            "ref_sizes": (None, [i]),
            "refh_mppi_rollout": (I, [E, M, S, f, f, f, f, u64, u64, d, i, i, I]),
            "refh_mppi_update": (I, [E, M, f, d, i, i, f, f, f, f, f, f, f, I]),
            "refh_mppi_verify": (I, [E, M, S, f, f, u64, u64, I, u, i, I]),
            "refh_spline_matrix": (I, [E, M, f]),
            "refh_cp_lower": (C.c_double, [C.c_uint, C.c_uint, C.c_double]),
            "refh_cp_upper": (C.c_double, [C.c_uint, C.c_uint, C.c_double]),
            "refh_pr_rollout": (I, [E, PR, S, f, f, f, i, u64, u64, d, d, I]),
            "refh_pr_candidates": (I, [E, PR, S, f, f, i, u64, u64, I, d, d]),
            "refh_env_step": (I, [E, I, f, S, f, I, I, C.c_float, I, I, u64, u64, I]),
            "refh_costs": (None, [E, M, PR, S, f]),
            "refc_device_count": (I, []),
            "refc_mppi_rollout": (I, [E, M, S, f, f, f, f, u64, f, i, i]),
            "refc_mppi_update": (I, [E, M, f, f, i, i, f, f, f, f, f, f, f]),
            "refc_mppi_verify": (I, [E, M, S, f, f, u64, u]),
            "refc_pr_rollout": (I, [E, PR, S, f, f, f, i, u64, f, f]),
            "refc_pr_update": (I, [PR, f, f, f, f, f, f, f, f, f, f, f]),
            "refc_pr_candidates": (I, [E, PR, S, f, f, f, i, u64, f, f]),
            "refc_mppi_time": (I, [E, M, S, I, I, I, d]),
            "refc_prmppi_time": (I, [E, PR, S, I, I, I, d]),
        }
        for n, (r, args) in protos.items():
            fn = getattr(L, n)
            fn.restype = r
            fn.argtypes = args
        _refs[variant] = L
    return _refs[variant]


# ---- convenience wrappers over Scenario objects -------------------------------------------

def _f(a):
    return _types().fptr(a)


def _d(a):
    return _types().dptr(a)


def _i(a):
    return _types().iptr(a)


def _u(a):
    return _types().uptr(a)


def _gate(sc) -> bool:
    """A gate-race scenario (its env is a dr_gate_env_config)."""
    return isinstance(sc.env, _types().dr_gate_env_config)


def gate_env_step(sc, true_theta, action, state, belief, update_belief=True, consider_branching=False, min_confidence=2.0, add_margin=False,
                  gate_margin=0.0, lose_on_opp_win=True, apply_noise=True, step=0, t=0, prec=32, impl="port"):
    """One gate-race environmentStep on a copy of `state`; returns (term, state', belief')."""
    a = _types()
    st = a.dr_gate_state.from_buffer_copy(state)
    bel = np.zeros(a.DR_MAX_THETA, np.float32)
    bel[: sc.n_theta] = belief
    act = np.ascontiguousarray(action, np.float32)
    if impl == "port":
        term = port().orc_gate_env_step(prec, C.byref(sc.env), true_theta, _f(act), C.byref(st), _f(bel), int(update_belief), int(consider_branching),
                                        min_confidence, int(add_margin), gate_margin, int(lose_on_opp_win), int(apply_noise), sc.seed, step, t)
    else:
        term = ref(impl).refh_env_step(C.byref(sc.env), true_theta, _f(act), C.byref(st), _f(bel), int(update_belief), int(consider_branching),
                                       min_confidence, int(lose_on_opp_win), int(apply_noise), sc.seed, step, t)
    return term, st, bel[: sc.n_theta].copy()


def gate_costs(sc, state, impl="port") -> np.ndarray:
    """(stateCost, finalCost) of a gate-race state."""
    out = np.zeros(4, np.float32)
    if impl == "port":
        port().orc_gate_costs(C.byref(sc.env), C.byref(sc.mppi), C.byref(state), _f(out))
        return out[:2]
    pc = _types().dr_prmppi_config()
    ref(impl).refh_costs(C.byref(sc.env), C.byref(sc.mppi), C.byref(pc), C.byref(state), _f(out))
    return np.array([out[0], out[3]], np.float32)


def nbp(sc) -> int:
    return sc.n_theta + 1


def mk(cfg) -> int:
    return cfg.n_knots if cfg.use_splines else cfg.n_timesteps


def sigma(cfg) -> np.ndarray:
    s = np.array([cfg.sampling_noise_dim[0], cfg.sampling_noise_dim[1]], dtype=np.float32)
    if not s.any():
        s[:] = cfg.sampling_noise
    return s


def mppi_noise(sc, step: int) -> np.ndarray:
    c = sc.mppi
    out = np.zeros((nbp(sc), mk(c), c.n_samples, 2), np.float32)
    port().orc_mppi_noise(sc.seed, step, nbp(sc), mk(c), c.n_samples, _f(sigma(c)), _f(out))
    return out


def pr_noise(sc, step: int) -> np.ndarray:
    c = sc.prmppi
    out = np.zeros((c.n_timesteps, c.n_samples, 2), np.float32)
    port().orc_pr_noise(sc.seed, step, c.n_timesteps, c.n_samples, _f(sigma(c)), _f(out))
    return out


def pr_thetas(sc, step: int, belief: np.ndarray) -> np.ndarray:
    out = np.zeros(sc.prmppi.P, np.int32)
    port().orc_pr_thetas(sc.seed, step, sc.prmppi.P, sc.n_theta, _f(np.ascontiguousarray(belief, np.float32)), _i(out))
    return out


def spline_matrix(cfg) -> np.ndarray:
    T, M = cfg.n_timesteps, cfg.n_knots
    B = np.zeros((T, M), np.float32)
    kn = np.array(cfg.knots[:M], np.int32)
    port().orc_spline_matrix(T, M, _i(kn), _f(B))
    return B


def mppi_rollout(sc, belief, nominal, noise, B, step, prec=32, impl="port", nthreads=0):
    """Returns costsTrue (n_theta, K) float64, branchUsed, branchTime (n_theta, K) int32."""
    c = sc.mppi
    K = c.n_samples
    ct = np.zeros((sc.n_theta, K), np.float64)
    bu = np.zeros((sc.n_theta, K), np.int32)
    bt = np.zeros((sc.n_theta, K), np.int32)
    belief = np.ascontiguousarray(belief, np.float32)
    nominal = np.ascontiguousarray(nominal, np.float32)
    noise = np.ascontiguousarray(noise, np.float32)
    Bm = np.ascontiguousarray(B if B is not None else np.zeros(1), np.float32)
    if impl == "port":
        fn = port().orc_gate_rollout if _gate(sc) else port().orc_mppi_rollout
        rc = fn(prec, C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(belief), _f(nominal), _f(noise), _f(Bm), sc.seed, step, _d(ct), _i(bu), _i(bt))
    else:
        rc = ref(impl).refh_mppi_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(belief), _f(nominal), _f(noise), _f(Bm), sc.seed, step,
                                         _d(ct), _i(bu), _i(bt), nthreads or os.cpu_count())
    assert rc == 0, rc
    return ct, bu, bt


def mppi_update(sc, belief, ct, bu, bt, noise, B, knots, prec=32, impl="port", blockorder=1, nthreads=0):
    """Returns (knots', dense, minCosts, nu, costs) like aggregate..clamp of the reference."""
    c = sc.mppi
    T, M, K, n = c.n_timesteps, mk(c), c.n_samples, nbp(sc)
    belief = np.ascontiguousarray(belief, np.float32)
    Bm = np.ascontiguousarray(B if B is not None else np.zeros(1), np.float32)
    if impl == "port":
        kn = np.ascontiguousarray(knots, np.float64).copy()
        dense = np.zeros((n, T, 2), np.float64)
        mins = np.zeros((n, M), np.float64)
        nu = np.zeros(n, np.float64)
        costs = np.zeros((n, K), np.float64)
        fn = port().orc_gate_update if _gate(sc) else port().orc_mppi_update
        fn(prec, C.byref(sc.env), C.byref(c), _f(belief), _d(np.ascontiguousarray(ct, np.float64)), _i(bu), _i(bt), _f(np.ascontiguousarray(noise, np.float32)),
           _f(Bm), _d(kn), _d(dense), _d(mins), _d(nu), _d(costs), blockorder)
    else:
        kn = np.ascontiguousarray(knots, np.float32).copy()
        dense = np.zeros((n, T, 2), np.float32)
        mins = np.zeros((n, M), np.float32)
        nu = np.zeros(n, np.float32)
        costs = np.zeros((n, K), np.float32)
        rc = ref(impl).refh_mppi_update(C.byref(sc.env), C.byref(c), _f(belief), _d(np.ascontiguousarray(ct, np.float64)), _i(bu), _i(bt),
                                        _f(np.ascontiguousarray(noise, np.float32)), _f(Bm), _f(kn), _f(dense), _f(mins), _f(nu), _f(costs),
                                        nthreads or os.cpu_count())
        assert rc == 0, rc
    return kn, dense, mins, nu, costs


def mppi_verify(sc, belief, plan, step, plan_id, prec=32, impl="port", nthreads=0):
    c = sc.mppi
    fc = np.zeros(c.n_timesteps, np.uint32)
    ft = np.zeros(c.n_verif_samples, np.int32)
    belief = np.ascontiguousarray(belief, np.float32)
    if impl == "port":
        th = np.zeros(c.n_verif_samples, np.int32)
        fn = port().orc_gate_verify if _gate(sc) else port().orc_mppi_verify
        fn(prec, C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(belief), _d(np.ascontiguousarray(plan, np.float64)), sc.seed, step, plan_id, _u(fc),
           _i(ft), _i(th))
        return fc, ft, th
    rc = ref(impl).refh_mppi_verify(C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(belief), _f(np.ascontiguousarray(plan, np.float32)), sc.seed,
                                    step, plan_id, _u(fc), _i(ft), nthreads or os.cpu_count())
    assert rc == 0, rc
    return fc, ft, None


def pr_rollout(sc, nom, rob, noise, thetas, step, prec=32, impl="port", nthreads=0):
    c = sc.prmppi
    P, K = c.P, c.n_samples
    cn = np.zeros((P, K, 2), np.float64)
    cr = np.zeros((P, K, 2), np.float64)
    thetas = np.ascontiguousarray(thetas, np.int32)
    noise = np.ascontiguousarray(noise, np.float32)
    if impl == "port":
        port().orc_pr_rollout(prec, C.byref(sc.env), C.byref(c), C.byref(sc.state), _d(np.ascontiguousarray(nom, np.float64)),
                              _d(np.ascontiguousarray(rob, np.float64)), _f(noise), _i(thetas), sc.seed, step, _d(cn), _d(cr))
    else:
        rc = ref(impl).refh_pr_rollout(C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(np.ascontiguousarray(nom, np.float32)),
                                       _f(np.ascontiguousarray(rob, np.float32)), _f(noise), _i(thetas), sc.seed, step, _d(cn), _d(cr),
                                       nthreads or os.cpu_count())
        assert rc == 0, rc
    return cn, cr


def pr_update(sc, cn, cr, noise, nom, rob, inv_temps, prec=32, blockorder=1):
    c = sc.prmppi
    T = c.n_timesteps
    cn = np.ascontiguousarray(cn, np.float64).copy()
    cr = np.ascontiguousarray(cr, np.float64).copy()
    mins = np.zeros(3, np.float64)
    c1, c2, nr = (np.zeros((T, 2), np.float64) for _ in range(3))
    nu = np.zeros(3, np.float64)
    port().orc_pr_update(prec, C.byref(c), _d(cn), _d(cr), _f(np.ascontiguousarray(noise, np.float32)), _d(np.ascontiguousarray(nom, np.float64)),
                         _d(np.ascontiguousarray(rob, np.float64)), _f(np.ascontiguousarray(inv_temps, np.float32)), _d(mins), _d(c1), _d(c2), _d(nr),
                         _d(nu), blockorder)
    return cn, cr, mins, c1, c2, nr, nu


def pr_candidates(sc, cand1, cand2, thetas, step, stream, prec=32, impl="port"):
    c = sc.prmppi
    full = np.zeros(2 * c.P, np.float64)
    safe = np.zeros(2 * c.P, np.float64)
    thetas = np.ascontiguousarray(thetas, np.int32)
    if impl == "port":
        port().orc_pr_candidates(prec, C.byref(sc.env), C.byref(c), C.byref(sc.state), _d(np.ascontiguousarray(cand1, np.float64)),
                                 _d(np.ascontiguousarray(cand2, np.float64)), _i(thetas), sc.seed, step, stream, _d(full), _d(safe))
    else:
        rc = ref(impl).refh_pr_candidates(C.byref(sc.env), C.byref(c), C.byref(sc.state), _f(np.ascontiguousarray(cand1, np.float32)),
                                          _f(np.ascontiguousarray(cand2, np.float32)), _i(thetas), sc.seed, step, stream, _d(full), _d(safe))
        assert rc == 0, rc
    return full, safe


S_PR_CAND_ENV = 8
S_PR_SAFE_ENV = 9


# ---- gradient path (FP64 forward-mode reference) ------------------------------------------

def nominal_cost(sc, state, belief, U, w6=None, dU=None, dW=None, B=None):
    """FP64 objective of the noise-free rollout of the control sequence U
    ((n_theta+1, M, 2)) and its directional derivative along (dU, dW).

    Returns (J, dJ, sig) with sig (n_theta, 3): steps rolled out, predTheta and
    branchingTime per hypothesis (-1 where incompatible)."""
    c = sc.mppi
    if B is None:
        B = spline_matrix(c) if c.use_splines else np.zeros((1, 1), np.float32)
    U = np.ascontiguousarray(U, np.float64)
    out = np.zeros(2, np.float64)
    sig = np.zeros((sc.n_theta, 3), np.int32)
    w = None if w6 is None else np.ascontiguousarray(w6, np.float64)
    du = None if dU is None else np.ascontiguousarray(dU, np.float64)
    dw = None if dW is None else np.ascontiguousarray(dW, np.float64)
    port().orc_nominal_cost(C.byref(sc.env), C.byref(c), C.byref(state), _f(np.ascontiguousarray(belief, np.float32)),
                            _f(np.ascontiguousarray(B, np.float32)), _d(U), None if w is None else _d(w), None if du is None else _d(du),
                            None if dw is None else _d(dw), _d(out), _i(sig))
    return float(out[0]), float(out[1]), sig
