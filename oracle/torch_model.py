"""TEST INFRASTRUCTURE (oracle). Not part of the product: only tests/ import it, as a
checker of the gradient path.

PyTorch FP64 autograd transcription of the objective that the gradient kernel
differentiates: an MPPI controller's noise-free rollout of its control sequence U
(the reference's fullRolloutKernel, src/kernels.cu:34-171, every noise source off),
per compatible hypothesis, averaged with the belief weights of
aggregateBranchCostsKernel (kernels.cu:175-217). The model is the reference's
StratRace environment step (include/environments/env_stratrace.h:711-894 and its
callees) and costs (include/costs.cuh:7-39), written line for line after the oracle's
C++ restatement (oracle/port/model.hpp, which cites the same reference lines) on 0-d
float64 tensors. Discrete decisions (argmin windows, clamps, branches, terminations,
lap counts, branching) are taken on the values and held, so torch.autograd gives the
exact gradient of the piecewise-smooth rollout with respect to U and the six cost
weights, in reverse mode: an independent check of both the CUDA adjoint and the
forward-mode dual-number oracle (oracle/port/grad.cpp).

Scalar tensors make this slow (about a second per 40-step rollout); it is meant for
small cases.
"""
from __future__ import annotations

import math

import numpy as np
import torch

NTS = 512
DIM = 2
WINDOW = 10  # env_stratrace_defs.h:40
DECAY = float(np.float32(0.97))  # include/config.h:30, a float constant
TERM_NONE, TERM_LOSE, TERM_WIN, TERM_OPP_WIN = 0, 1, 2, 3
F64 = torch.float64


def _v(x) -> float:
    return float(x.item()) if torch.is_tensor(x) else float(x)


def _t(x) -> torch.Tensor:
    return x if torch.is_tensor(x) else torch.tensor(float(x), dtype=F64)


def _sqrt(x):
    # value sqrt, derivative 0 at 0 (as the dual-number oracle), not inf
    return torch.sqrt(_t(x)) if _v(x) > 0.0 else _t(x) * 0.0


def _fmin(a, b):
    return a if _v(a) <= _v(b) else b


def _fmax(a, b):
    return a if _v(a) >= _v(b) else b


def _floor(x) -> float:
    return math.floor(_v(x))


def _copysign(a, b):
    # |a| with the sign of b; the derivative follows the sign applied to a
    return a if math.copysign(1.0, _v(a)) == math.copysign(1.0, _v(b)) else -a


class Env:
    """dr_env_config in float64 (oracle/port/model.hpp Env); grids padded by one wrap sample."""

    def __init__(self, c):
        self.nopp, self.nth = int(c.n_opp), int(c.n_theta)
        self.dt, self.droneRadius = float(c.dt), float(c.drone_radius)
        self.maxSpeed = [float(v) for v in c.max_speed]
        self.maxAccel = [float(v) for v in c.max_accel]
        self.trackWidth, self.nWinLaps = float(c.track_width), int(c.n_win_laps)
        self.kP, self.kV = float(c.kP), float(c.kV)
        self.maxOppLatDistFact, self.L = float(c.max_opp_lat_dist_fact), float(c.track_length)
        oc = c.opp_configs
        self.s1 = [[float(oc[th].s1[o]) for o in range(max(1, self.nopp))] for th in range(self.nth)]
        self.s2 = [[float(oc[th].s2[o]) for o in range(max(1, self.nopp))] for th in range(self.nth)]
        self.s3 = [[float(oc[th].s3[o]) for o in range(max(1, self.nopp))] for th in range(self.nth)]
        self.speedScale = [[float(oc[th].speed_scale[o]) for o in range(max(1, self.nopp))] for th in range(self.nth)]
        self.actionNoise = [[float(oc[th].action_noise[o]) for o in range(max(1, self.nopp))] for th in range(self.nth)]
        p = np.array(c.p_grid[: NTS * 2], np.float64).reshape(NTS, 2)
        t = np.array(c.t_grid[: NTS * 2], np.float64).reshape(NTS, 2)
        k = np.array(c.kappa_grid[:NTS], np.float64)
        self.p = np.vstack([p, p[:1]]).tolist()
        self.t = np.vstack([t, t[:1]]).tolist()
        self.kappa = np.concatenate([k, k[:1]]).tolist()


class State:
    def __init__(self, s, na: int):
        self.pos = [_t(s.pos[i]) for i in range(na * 2)]
        self.vel = [_t(s.vel[i]) for i in range(na * 2)]
        self.S = [_t(s.S[a]) for a in range(na)]
        self.lat = [_t(s.lat_dist[a]) for a in range(na)]
        self.laps = [int(s.laps[a]) for a in range(na)]


def find_confident(belief, nth: int, thr: float) -> int:  # state.h:93-115
    for th in range(nth):
        if _v(belief[th]) > thr:
            return th + 1
    return 0


def _sample2(arr, s, L):  # sampleTrackArray<true>, :53-67
    s = s / L
    s = s - _floor(s)
    idx_f = s * NTS
    i0 = int(_v(idx_f))
    i1 = (i0 + 1) % NTS
    t = idx_f - i0
    return [(1.0 - t) * arr[i0][d] + t * arr[i1][d] for d in range(DIM)]


def _sample1(arr, s, L):  # sampleTrackArray<false>
    s = s / L
    s = s - _floor(s)
    idx_f = s * NTS
    i0 = int(_v(idx_f))
    i1 = (i0 + 1) % NTS
    t = idx_f - i0
    return (1.0 - t) * arr[i0] + t * arr[i1]


def _norm_speed(env, s):  # sampleNormalizedSpeed, :69-76
    o = _sample2(env.t, s, env.L)
    inv = 1.0 / _sqrt(o[0] * o[0] + o[1] * o[1])
    return [o[0] * inv, o[1] * inv]


def project(env, pos, prevS):  # fastProjectOnTrack<false>, :88-162 -> (S, latDist)
    ps = prevS / env.L
    ps = ps - _floor(ps)
    idxPrev = int(_v(ps) * NTS)
    P = env.p
    px, py = _v(pos[0]), _v(pos[1])

    def sqd(i):
        return (P[i][0] - px) * (P[i][0] - px) + (P[i][1] - py) * (P[i][1] - py)

    best = (idxPrev - WINDOW + NTS) % NTS
    bestSq = sqd(best)
    for off in range(NTS - WINDOW + 1, NTS + WINDOW + 1):
        i = (idxPrev + off) % NTS
        d = sqd(i)
        if d < bestSq:
            bestSq, best = d, i
    bestSegSq = math.inf
    bestS = closest = segSq = None
    for seg in (-1, 0):
        a = (best + seg + NTS) % NTS
        b = (a + 1) % NTS
        abx, aby = P[b][0] - P[a][0], P[b][1] - P[a][1]
        sqAB = abx * abx + aby * aby
        t = _t(0.0)
        if sqAB > 1e-12:
            t = ((pos[0] - P[a][0]) * abx + (pos[1] - P[a][1]) * aby) / sqAB
            t = _fmax(_t(0.0), _fmin(t, _t(1.0)))
        projx = P[a][0] + t * abx
        projy = P[a][1] + t * aby
        dx, dy = pos[0] - projx, pos[1] - projy
        sq = dx * dx + dy * dy
        if _v(sq) < bestSegSq:
            bestSegSq = _v(sq)
            segSq = sq
            bestS = (a + t) / NTS * env.L
            closest = (projx, projy)
    tang = _sample2(env.t, bestS, env.L)
    cross = -tang[1] * (pos[0] - closest[0]) + tang[0] * (pos[1] - closest[1])
    return bestS, _copysign(_sqrt(segSq), cross)


def update_belief(env, belief, oppAction, nom):  # :166-222; nom[th][o] = (x, y)
    total = _t(0.0)
    sig_env = 0.2
    out = list(belief)
    for th in range(env.nth):
        ll = _t(0.0)
        for o in range(env.nopp):
            n = nom[th][o]
            obs = oppAction[o]
            sqA = n[0] * n[0] + n[1] * n[1]
            scale = _t(1.0)
            if _v(sqA) > env.maxAccel[o + 1] * env.maxAccel[o + 1]:
                scale = env.maxAccel[o + 1] / _sqrt(sqA)
            sqD = _t(0.0)
            for d in range(DIM):
                dx = obs[d] - n[d] * scale
                sqD = sqD + dx * dx
            an = env.actionNoise[th][o]
            sqS = sig_env * sig_env + an * an
            ll = ll + (-0.5) * sqD / sqS - DIM * 0.5 * math.log(2.0 * math.pi) - DIM * 0.5 * math.log(sqS)
        out[th] = out[th] * torch.exp(ll)
        total = total + out[th]
    if _v(total) < 1e-20:
        return [_t(1.0 / env.nth) for _ in range(env.nth)]
    return [out[th] / total for th in range(env.nth)]


def boundary_dist(s, env, loseOnOppWin: bool):  # trackBoundaryDist, :226-244
    if loseOnOppWin:
        for o in range(1, env.nopp + 1):
            if s.laps[o] >= env.nWinLaps:
                return _t(-1.0)
    minSq = None
    for o in range(1, env.nopp + 1):
        dx, dy = s.pos[2 * o] - s.pos[0], s.pos[2 * o + 1] - s.pos[1]
        sq = dx * dx + dy * dy
        minSq = sq if minSq is None else _fmin(minSq, sq)
    return _fmin(_sqrt(minSq) - env.droneRadius, env.trackWidth - torch.abs(s.lat[0]))


def is_winner(s, env) -> bool:  # :252-265
    if s.laps[0] >= env.nWinLaps:
        return True
    return any(abs(_v(s.lat[o])) > env.trackWidth - env.droneRadius for o in range(1, env.nopp + 1))


def is_opp_winner(s, env) -> bool:  # :267-274
    return any(s.laps[o] >= env.nWinLaps for o in range(1, env.nopp + 1))


def _advance(s, env, a):  # :277-280
    return s.S[a] / env.L + s.laps[a]


def sdot(i, s, env):  # computeSdot, :302-315
    tg = _norm_speed(env, s.S[i])
    k = _sample1(env.kappa, s.S[i], env.L)
    metric = 1 - k * s.lat[i]
    if abs(_v(metric)) < 1e-12:
        metric = _t(math.copysign(1e-12, _v(metric)))
    return (tg[0] * s.vel[2 * i] + tg[1] * s.vel[2 * i + 1]) / metric


def opp_target(iOpp, s, env, th):  # computeOppTargetLatDist, :318-461 -> (latDis, speedGoal)
    L = env.L
    iAhead, dA = 0, s.S[0] - s.S[iOpp]
    if _v(dA) < 0:
        dA = dA + L
    for j in range(1, env.nopp + 1):
        if j != iOpp:
            d = s.S[j] - s.S[iOpp]
            if _v(d) < 0:
                d = d + L
            if _v(d) < _v(dA):
                dA, iAhead = d, j
    iBehind, dB = 0, s.S[0] - s.S[iOpp]
    if _v(dB) > 0:
        dB = dB - L
    for j in range(1, env.nopp + 1):
        if j != iOpp:
            d = s.S[j] - s.S[iOpp]
            if _v(d) > 0:
                d = d - L
            if _v(d) > _v(dB):
                dB, iBehind = d, j
    latDis = _t(0.0)
    sd_i = sdot(iOpp, s, env)
    base = env.speedScale[th][iOpp - 1] * env.maxSpeed[iOpp]
    goal = _t(base)
    s1, s2, s3 = env.s1[th][iOpp - 1], env.s2[th][iOpp - 1], env.s3[th][iOpp - 1]
    for k in (0, 1):
        j = iAhead if k else iBehind
        dS = dA if k else dB
        dE = s.lat[j] - s.lat[iOpp]
        tg_j = _norm_speed(env, s.S[j])
        sd_j = sdot(j, s, env)
        tol = env.maxSpeed[j] * 0.3
        block = _v(dS) < 0 and _v(dS) > -env.L * 0.25 and _v(sd_j) + tol > _v(sd_i)
        overtake = _v(sd_i) > _v(sd_j) and abs(_v(dE)) < s1
        factor = torch.exp(-s2 * dS * dS)
        if block:
            latDis = latDis + s.lat[j] * (1 - torch.exp(-s3 * (sd_j + tol - sd_i))) * factor
        if overtake:
            latDis = latDis + (s.lat[j] - math.copysign(s1, _v(dE))) * factor
            oppLong = s.vel[2 * j] * tg_j[0] + s.vel[2 * j + 1] * tg_j[1]
            if _v(dS) < 3 * env.droneRadius:
                goal = _fmin(goal, 0.7 * oppLong)
            elif _v(dS) < 6 * env.droneRadius and s1 > 1e-6:
                lf = torch.abs(dE) / s1
                goal = _fmin(goal, lf * oppLong + (1.0 - lf) * base)
    mx = env.trackWidth - env.droneRadius * env.maxOppLatDistFact
    latDis = _fmax(_t(-mx), _fmin(_t(mx), latDis))
    return latDis, goal


def opp_action(iOpp, s, env, th):  # computeOpponentAction, :611-706
    maxA, dt = env.maxAccel[iOpp], env.dt
    latRaw, goal = opp_target(iOpp, s, env, th)
    sn = s.S[iOpp]
    pc = _sample2(env.p, sn, env.L)
    tg = _norm_speed(env, sn)
    kap = _sample1(env.kappa, sn, env.L)
    nrm = [-tg[1], tg[0]]
    px, py = s.pos[2 * iOpp], s.pos[2 * iOpp + 1]
    vx, vy = s.vel[2 * iOpp], s.vel[2 * iOpp + 1]
    e_n = (px - pc[0]) * nrm[0] + (py - pc[1]) * nrm[1]
    v_t = vx * tg[0] + vy * tg[1]
    v_n = vx * nrm[0] + vy * nrm[1]
    e_max = env.trackWidth - env.droneRadius * 1.2
    metric = 1.0 - kap * e_n
    if abs(_v(metric)) < 1e-6:
        metric = _t(math.copysign(1e-6, _v(metric)))
    a_c = v_t * v_t * kap / metric
    a_lat = _fmax(maxA - torch.abs(a_c), _t(maxA * 0.2))
    latDis = _fmax(_t(-e_max), _fmin(_t(e_max), latRaw))
    e_err = latDis - e_n
    d_pos = _fmax(e_max - e_n, _t(0.001))
    d_neg = _fmax(e_max + e_n, _t(0.001))
    if _v(v_n) > 0 and _v(v_n * v_n) > _v(1.8 * a_lat * d_pos):
        a_n = -a_lat
    elif _v(v_n) < 0 and _v(v_n * v_n) > _v(1.8 * a_lat * d_neg):
        a_n = a_lat
    elif abs(_v(e_err)) < 0.02:
        kp = a_lat / 0.02
        a_n = kp * e_err - 2.0 * _sqrt(kp) * v_n
        a_n = _fmax(-a_lat, _fmin(a_lat, a_n))
    else:
        stop_d = v_n * v_n / (2.0 * a_lat)
        toward = (_v(e_err) > 0 and _v(v_n) > 0) or (_v(e_err) < 0 and _v(v_n) < 0)
        decel = toward and _v(stop_d) >= abs(_v(e_err)) * 0.95
        a_n = a_lat if _v(e_err) > 0 else -a_lat
        if decel:
            a_n = -a_n
        v_next = v_n + a_n * dt
        if _v(v_next) > 0:
            v_safe = _sqrt(2.0 * a_lat * d_pos)
            if _v(v_next) > _v(v_safe):
                a_n = (v_safe - v_n) / dt
        else:
            v_safe = _sqrt(2.0 * a_lat * d_neg)
            if -_v(v_next) > _v(v_safe):
                a_n = (-v_safe - v_n) / dt
    a_tot = _fmax(_t(-maxA), _fmin(_t(maxA), a_n + a_c))
    a_tmax = _sqrt(_fmax(maxA * maxA - a_tot * a_tot, _t(0.0)))
    k_eff = kap / (1.0 - kap * latDis + 1e-6)
    path = _fmin(goal, _sqrt(maxA / _fmax(torch.abs(k_eff), _t(1e-12))))
    if abs(_v(a_n)) > _v(a_lat) * 0.5:
        path = path * _fmax(_t(0.4), 1.5 - torch.abs(a_n) / a_lat)
    a_t = env.kV * (path - v_t) - v_n * kap * v_t / metric
    a_t = _fmax(-a_tmax, _fmin(a_tmax, a_t))
    return [a_t * tg[0] + a_tot * nrm[0], a_t * tg[1] + a_tot * nrm[1]]


def env_step(t, trueTheta, env, ego, s, bs, minConf):
    """environmentStep<updateBelief, considerBranching, loseOnOppWin = true>, noise off,
    every hypothesis' opponent action (:711-894). bs = [belief list, predTheta,
    branchingTime] is updated in place; returns (term, branched)."""
    na = env.nopp + 1
    prevS = [_v(x) for x in s.S]
    acts = [list(ego)]
    nom = [[None] * env.nopp for _ in range(env.nth)]
    for o in range(1, env.nopp + 1):
        for th in range(env.nth):
            nom[th][o - 1] = opp_action(o, s, env, th)
        acts.append(list(nom[trueTheta][o - 1]))
    for a in range(na):
        sq = acts[a][0] * acts[a][0] + acts[a][1] * acts[a][1]
        if _v(sq) > env.maxAccel[a] * env.maxAccel[a]:
            f = env.maxAccel[a] / _sqrt(sq)
            acts[a] = [acts[a][0] * f, acts[a][1] * f]
    for a in range(na):
        for d in range(DIM):
            s.pos[a * 2 + d] = s.pos[a * 2 + d] + env.dt * s.vel[a * 2 + d]
    for a in range(na):
        s.S[a] = s.S[a] + env.dt * sdot(a, s, env)
    for a in range(na):
        for d in range(DIM):
            s.vel[a * 2 + d] = s.vel[a * 2 + d] + env.dt * acts[a][d]
    for a in range(na):
        sq = s.vel[2 * a] * s.vel[2 * a] + s.vel[2 * a + 1] * s.vel[2 * a + 1]
        if _v(sq) > env.maxSpeed[a] * env.maxSpeed[a]:
            sc = env.maxSpeed[a] / _sqrt(sq)
            s.vel[2 * a] = s.vel[2 * a] * sc
            s.vel[2 * a + 1] = s.vel[2 * a + 1] * sc
    for a in range(na):
        s.S[a], s.lat[a] = project(env, s.pos[2 * a:2 * a + 2], s.S[a])
    for a in range(na):
        if _v(s.S[a]) < prevS[a] - env.L * 0.5:
            s.laps[a] += 1
        if _v(s.S[a]) > prevS[a] + env.L * 0.5:
            s.laps[a] -= 1
    bs[0] = update_belief(env, bs[0], acts[1:], nom)
    branched = False
    npred = find_confident(bs[0], env.nth, minConf)
    if bs[1] == 0 and npred != 0:
        bs[1], bs[2], branched = npred, t + 1, True
    if _v(boundary_dist(s, env, True)) < env.droneRadius:
        return TERM_LOSE, branched
    if is_winner(s, env):
        return TERM_WIN, branched
    return TERM_NONE, branched


def state_cost(s, env, w, collDistFactor, thrFactor):  # stateCost, costs.cuh:7-28; w = 6 weights
    cost = _t(0.0)
    bd = boundary_dist(s, env, False)
    if _v(bd) < thrFactor * env.droneRadius:
        cost = cost + w[0] * torch.pow(bd / env.droneRadius, 2.0)
    if _v(bd) < env.droneRadius * collDistFactor:
        cost = cost + w[1]
    if is_opp_winner(s, env):
        cost = cost + w[3]
    if is_winner(s, env):
        cost = cost - w[2]
    return cost


def final_cost(s, env, w):  # finalCost, costs.cuh:31-39
    cost = -w[4] * _advance(s, env, 0)
    if _v(w[5]) != 0.0:
        mx = None
        for o in range(1, env.nopp + 1):
            v = _advance(s, env, o)
            mx = v if mx is None else _fmax(mx, v)
        cost = cost + w[5] * mx
    return cost


def nominal_objective(env_cfg, mppi_cfg, state0, belief0, U, w6, B=None):
    """J(U, w6) of oracle/port/grad.cpp:orc_nominal_cost as a torch graph.

    U: float64 tensor (n_theta + 1, M, 2); w6: float64 tensor (6,) in the order
    boundary_cost, outside_cost, win_cost, opp_win_cost, final_adv_weight,
    final_opp_adv_weight; B: the T x M spline basis (float32 values) in spline mode."""
    env = Env(env_cfg)
    c = mppi_cfg
    T = int(c.n_timesteps)
    spl = bool(c.use_splines)
    M = int(c.n_knots) if spl else T
    minConf = float(np.float32(c.min_confidence))
    coll, thr = float(np.float32(c.coll_dist_factor)), float(np.float32(c.boundary_threshold_factor))
    w = [w6[i] for i in range(6)]
    b0 = [float(np.float32(x)) for x in belief0[: env.nth]]
    Bm = None if not spl else np.asarray(B, np.float32).astype(np.float64).reshape(T, M)
    pred0 = find_confident(b0, env.nth, minConf)
    bt0 = -1 if pred0 == 0 else 0
    num, den = _t(0.0), 0.0
    for th in range(env.nth):
        if pred0 != 0 and pred0 != th + 1:
            continue
        s = State(state0, env.nopp + 1)
        bs = [[_t(x) for x in b0], pred0, bt0]
        cost, decay, tOrigin = _t(0.0), 1.0, 0
        for t in range(T):
            local, b = t - tOrigin, bs[1]
            if spl:
                ego = [_spline(Bm[local], U[b, :, d]) for d in range(DIM)]
            else:
                ego = [U[b, local, 0], U[b, local, 1]]
            term, branched = env_step(t, th, env, ego, s, bs, minConf)
            if branched:
                tOrigin = t + 1
            cost = cost + state_cost(s, env, w, coll, thr) * decay
            decay *= DECAY
            if term != TERM_NONE:
                break
        cost = cost + final_cost(s, env, w)
        if not math.isfinite(_v(cost)):
            continue
        num = num + b0[th] * cost
        den += b0[th]
    if den <= 1e-30:
        return _t(math.inf)
    return num / den


def _spline(row, u):
    # sum over knots in knot order, as the oracle's loop (a serial sum)
    acc = _t(0.0)
    for m in range(len(row)):
        acc = acc + float(row[m]) * u[m]
    return acc


def nominal_grad(env_cfg, mppi_cfg, state0, belief0, U, w6, B=None):
    """(J, dJ/dU, dJ/dw6) in float64 by reverse-mode autograd."""
    Ut = torch.tensor(np.asarray(U, np.float64), dtype=F64, requires_grad=True)
    Wt = torch.tensor(np.asarray(w6, np.float64), dtype=F64, requires_grad=True)
    J = nominal_objective(env_cfg, mppi_cfg, state0, belief0, Ut, Wt, B)
    if not math.isfinite(_v(J)):
        return _v(J), np.zeros_like(np.asarray(U, np.float64)), np.zeros(6)
    J.backward()
    return _v(J), Ut.grad.numpy().copy(), Wt.grad.numpy().copy()
