"""Test helpers: small scenarios and the controller step composed from oracle pieces."""
from __future__ import annotations

import ctypes as C

import numpy as np

from conftest import O, drb

S = drb.scenarios
abi = drb.abi


def zero_env_noise(sc):
    """Turn off every in-rollout noise source (opponent action noise, action/pos/speed
    noise): the reference kernels draw those from curand, which cannot be injected."""
    for th in range(abi.DR_MAX_THETA):
        for o in range(abi.DR_MAX_OPP):
            sc.env.opp_configs[th].action_noise[o] = 0.0
    sc.env.action_noise_level = 0.0
    sc.env.pos_noise_level = 0.0
    sc.env.speed_noise_level = 0.0
    return sc


def small_mppi(use_splines: bool, K=512, T=40, M=10, n_verif=1024, seed=7, noise=True):
    sc = S.strat_race(use_splines=use_splines, K=K, T=T, n_verif=n_verif)
    sc.seed = seed
    if use_splines:
        sc.mppi = S.make_mppi(K=K, T=T, use_splines=True, M=M, n_verif_samples=n_verif, verif_horizon=min(30, T))
    else:
        sc.mppi = S.make_mppi(K=K, T=T, use_splines=False, inv_temperature=10, sampling_noise=1.5, coll_dist_factor=1.3, final_adv_weight=500,
                              boundary_cost=50, boundary_threshold_factor=1.7, outside_cost=1e6, win_cost=1e6, opp_win_cost=1e5,
                              n_verif_samples=n_verif, verif_horizon=min(30, T))
    if not noise:
        zero_env_noise(sc)
    return sc


def mppi_ctl(sc, nominal=None, exact_verify=False):
    """exact_verify: the verification's exact flavour, whose per-sample results equal the
    oracle's (tests that compare a step's plan choice or failure counts with the oracle)."""
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed, nominal=nominal)
    if exact_verify:
        ctl.set_verify_exact(True)
    return ctl


def random_nominal(sc, rng, scale=0.8):
    c = sc.mppi
    return rng.normal(0, scale, (sc.n_theta + 1, c.n_timesteps, 2)).astype(np.float32)


def knots_of(ctl) -> np.ndarray:
    return ctl.knots()


class OracleMPPI:
    """MPPIController::getControl (src/mppi_controller.cu:250-466) composed from the
    oracle port's pieces, in FP32 or FP64."""

    def __init__(self, sc, nominal=None, prec=32):
        self.sc = sc
        c = sc.mppi
        self.prec = prec
        self.T, self.M, self.nbp = c.n_timesteps, O.mk(c), sc.n_theta + 1
        self.B = O.spline_matrix(c) if c.use_splines else None
        nom = np.zeros((self.nbp, self.T, 2)) if nominal is None else np.asarray(nominal, np.float64).reshape(self.nbp, self.T, 2)
        self.h_nominal = nom.copy()
        self.dense = nom.copy()
        self.prev = nom.copy()
        self.knots = np.zeros((self.nbp, self.M, 2)) if c.use_splines else nom.copy()
        self.lam = float(c.inv_temperature)
        self.step = 0
        self.pend = None

    def get_control(self, state, belief):
        sc, c = self.sc, self.sc.mppi
        if self.pend is not None:
            b, use_new = self.pend
            src = (self.dense if use_new else self.prev).copy()
            src[b, :-1] = src[b, 1:]
            src[b, -1] = 0
            self.prev = src.copy()
            self.dense = src.copy()
            if c.use_splines:
                kn = np.ascontiguousarray(self.knots, np.float64)
                O.port().orc_shift_spline(C.byref(c), O._f(self.B), O._d(kn), b, self.prec)
                self.knots = kn
            else:
                self.knots = src.copy()
        old_state = sc.state
        sc.state = state
        cfg_lam = c.inv_temperature
        c.inv_temperature = self.lam
        try:
            noise = O.mppi_noise(sc, self.step)
            kn32 = np.ascontiguousarray(self.knots, np.float32)
            ct, bu, bt = O.mppi_rollout(sc, belief, kn32, noise, self.B, self.step, prec=self.prec)
            knots, dense, mins, nu, costs = O.mppi_update(sc, belief, ct, bu, bt, noise, self.B, self.knots, prec=self.prec)
            self.knots = knots.reshape(self.nbp, self.M, 2)
            self.dense = dense.reshape(self.nbp, self.T, 2)
            if c.verify:
                fc_new, _, _ = O.mppi_verify(sc, belief, self.dense, self.step, 0, prec=self.prec)
                fc_old, _, _ = O.mppi_verify(sc, belief, self.prev, self.step, 1, prec=self.prec)
            else:
                fc_new = fc_old = np.zeros(self.T, np.uint32)
        finally:
            sc.state = old_state
            c.inv_temperature = cfg_lam
        V = c.n_verif_samples
        cert = -1.0
        tn = to = 0
        for t in range(self.T if c.verify else 0):
            tn += int(fc_new[t])
            to += int(fc_old[t])
            e1 = O.port().orc_cp_upper(tn, V, float(np.float32(c.beta)) / 2.0)
            e2 = O.port().orc_cp_lower(to, V, float(np.float32(c.beta)) / 2.0)
            cert = max(cert, e1 - e2)
        use_new = cert < float(np.float32(c.max_verif_eps)) if c.verify else True
        chosen = self.dense if use_new else self.prev
        self.h_nominal = chosen.copy()
        bidx = 0
        for th in range(sc.n_theta):
            if belief[th] > np.float32(c.min_confidence):
                bidx = th + 1
                break
        action = np.float32(self.h_nominal[bidx, 0])
        used_nu = np.float32(nu[bidx])
        if used_nu > np.float32(np.float32(c.max_nu) * np.float32(c.n_samples)):
            self.lam = float(np.float32(self.lam) * np.float32(0.9))
        elif used_nu < np.float32(np.float32(c.min_nu) * np.float32(c.n_samples)):
            self.lam = float(np.float32(self.lam) * np.float32(1.2))
        self.h_nominal[bidx, :-1] = self.h_nominal[bidx, 1:]
        self.h_nominal[bidx, -1] = 0
        self.pend = (bidx, use_new)
        self.step += 1
        return action, dict(use_new=use_new, cert=cert, fc_new=fc_new, fc_old=fc_old, nu=nu, mins=mins, bidx=bidx)


def small_gate(use_splines: bool, K=512, T=40, n_verif=1024, seed=7, noise=True, agent=0, gap=None):
    """A small gate-race case; noise=False turns off the PID action noise (the reference's
    kernels draw it from curand). gap (fraction of a lap): put the ego that far behind the
    opponent on its raceline, both at 2 m/s."""
    sc = S.gate_race(agent=agent, K=K, T=T, use_splines=use_splines, n_verif=n_verif, action_noise=0.5 if noise else 0.0)
    sc.seed = seed
    if gap is not None:
        n = sc.track.shape[1]
        opp_u = float(np.float32(sc.state.S[2] if sc.state.S[2] >= 0 else sc.state.S[0]))
        st = S.gate_state(sc.track, [opp_u - gap, opp_u], 0, list(sc.state.gates), speed=2.0)
        sc.state = st
    return sc


def toward_opponent_plan(sc, accel=6.0):
    """A dense plan accelerating the ego straight at the opponent on every branch: many
    verification samples end in a collision."""
    st = sc.state
    me = int(sc.env.i_mppi)
    d = np.array([st.pos[2 * (1 - me)] - st.pos[2 * me], st.pos[2 * (1 - me) + 1] - st.pos[2 * me + 1]], np.float64)
    d = d / np.linalg.norm(d) * accel
    return np.broadcast_to(d, (sc.n_theta + 1, sc.mppi.n_timesteps, 2)).astype(np.float32).copy()
