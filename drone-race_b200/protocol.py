"""The reference's configuration / result wire protocol, so that its Python front-end
(python-src/protocol.py, ZMQRecv.runSim) drives this implementation unchanged.

Framing (include/protocol.h:26-142, python-src/protocol.py:13-161): little-endian int32
and float32 scalars; an array is an int32 length followed by float32 elements (integer
arrays travel as floats too). Headers are decoded in the order of
src/environments/env_stratrace.cpp:135-226 (environment), src/config.cpp:5-115
(controller) and env_stratrace.cpp:98-118 (initial state), with the same checks:
message kind, compile-time sizes (here: the sizes this build supports), array lengths,
buffer underflow and trailing bytes.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

from . import abi
from .track import TrackGrids

MSG_HEADER, MSG_STATE, MSG_EVENT, MSG_DONE = 0, 1, 2, 3  # protocol.h:9-15
EVT_OUTSIDE, EVT_WINNER, EVT_OPP_WINNER, EVT_TRUNCATED = 0, 1, 2, 3  # protocol.h:17-23
CONT_MPPI, CONT_PRMPPI = 0, 1  # config.h:66-70
ENV_DRONERACE, ENV_HIDDENOBS, ENV_STRATRACE = 0, 1, 2  # config.h:71-76


class ProtocolError(RuntimeError):
    pass


class Reader:
    """include/protocol.h:26-108."""

    def __init__(self, buf: bytes):
        self.buf = memoryview(buf)
        self.off = 0

    def _take(self, n: int) -> memoryview:
        if self.off + n > len(self.buf):
            raise ProtocolError("failed to read scalar from buffer (underflow)")
        m = self.buf[self.off : self.off + n]
        self.off += n
        return m

    def int32(self) -> int:
        return struct.unpack("<i", self._take(4))[0]

    def float32(self) -> float:
        return struct.unpack("<f", self._take(4))[0]

    def array(self, expect: int | None = None, at_most: int | None = None) -> np.ndarray:
        n = self.int32()
        if n < 0:
            raise ProtocolError(f"Negative array length: {n}")
        if expect is not None and n != expect:
            raise ProtocolError(f"Wrong size when reading array: read length {n}, allocated length {expect}")
        if at_most is not None and n > at_most:
            raise ProtocolError(f"Wrong size when reading array: read length {n}, allocated length {at_most}")
        return np.frombuffer(self._take(4 * n), dtype="<f4").astype(np.float32)

    def finished(self) -> None:
        if self.off != len(self.buf):
            raise ProtocolError("Header not fully parsed")


class Writer:
    """include/protocol.h:111-142."""

    def __init__(self):
        self.parts: list[bytes] = []

    def int32(self, v: int) -> None:
        self.parts.append(struct.pack("<i", int(v)))

    def float32(self, v: float) -> None:
        self.parts.append(struct.pack("<f", float(v)))

    def array(self, a) -> None:
        a = np.asarray(a, dtype="<f4").ravel()
        self.int32(a.size)
        self.parts.append(a.tobytes())

    def bytes(self) -> bytes:
        return b"".join(self.parts)


@dataclass
class EnvHeader:
    env: abi.dr_env_config
    grids: TrackGrids
    seed: int
    true_theta: int
    model_sizes: list[int]


def unpack_env(buf: bytes) -> EnvHeader:
    """Env::unpackEnvConfig (env_stratrace.cpp:135-226)."""
    r = Reader(buf)
    if (k := r.int32()) != MSG_HEADER:
        raise ProtocolError(f"Expected header message type for environment config (type {MSG_HEADER}) but got type {k} instead")
    if (ek := r.int32()) != ENV_STRATRACE:
        raise ProtocolError(f"Environment kind mismatch: received kind {ek}, but this build implements ENV_STRATRACE ({ENV_STRATRACE})")
    n_factors = r.int32()
    if n_factors != 1:
        raise ProtocolError(f"Received config for {n_factors} environment parameters but this build supports one parameter factor")
    sizes = [int(x) for x in r.array()]
    n_theta = sizes[0] if sizes else 0
    if not 1 <= n_theta <= abi.DR_MAX_THETA:
        raise ProtocolError(f"Received invalid model size {n_theta} (supported: 1..{abi.DR_MAX_THETA})")
    e = abi.dr_env_config()
    e.n_theta = n_theta
    amin, amax = r.array(2), r.array(2)
    n_opp, dim = r.int32(), r.int32()
    e.dt = r.float32()
    e.send_states = r.int32()
    if not 1 <= n_opp <= abi.DR_MAX_OPP:
        raise ProtocolError(f"Received config for {n_opp} opponents (supported: 1..{abi.DR_MAX_OPP})")
    if dim != abi.DR_DIM:
        raise ProtocolError(f"Received config for dimension {dim} but DIM is {abi.DR_DIM}")
    e.n_opp = n_opp
    na = n_opp + 1
    for d in range(2):
        e.arena_min[d] = float(amin[d])
        e.arena_max[d] = float(amax[d])
    e.drone_radius = r.float32()
    e.pos_noise_level = r.float32()
    e.speed_noise_level = r.float32()
    e.action_noise_level = r.float32()
    ms, ma = r.array(na), r.array(na)
    for a in range(na):
        e.max_speed[a] = float(ms[a])
        e.max_accel[a] = float(ma[a])
    nts = r.int32()
    if nts != abi.DR_N_TRACK_SAMPLES:
        raise ProtocolError(f"Received config for {nts} track samples but N_TRACK_SAMPLES is {abi.DR_N_TRACK_SAMPLES}")
    e.track_width = r.float32()
    e.n_win_laps = r.int32()
    seed = r.int32()
    ib = r.array(n_theta)
    for th in range(n_theta):
        e.init_belief[th] = float(ib[th])
    for th in range(n_theta):
        oc = e.opp_configs[th]
        for name in ("s1", "s2", "s3", "speed_scale", "action_noise"):
            arr = r.array(n_opp)
            for o in range(n_opp):
                getattr(oc, name)[o] = float(arr[o])
    true_theta = r.int32()
    e.kP = r.float32()
    e.kV = r.float32()
    e.max_opp_lat_dist_fact = r.float32()
    e.track_length = r.float32()
    p = r.array(2 * nts).reshape(nts, 2).copy()
    dp = r.array(2 * nts).reshape(nts, 2).copy()
    t = r.array(2 * nts).reshape(nts, 2).copy()
    kap = r.array(nts).copy()
    r.finished()
    grids = TrackGrids(float(e.track_length), p, dp, t, kap)
    e.p_grid = abi.fptr(grids.p_grid)
    e.dp_grid = abi.fptr(grids.dp_grid)
    e.t_grid = abi.fptr(grids.t_grid)
    e.kappa_grid = abi.fptr(grids.kappa_grid)
    return EnvHeader(e, grids, seed, true_theta, sizes)


def pack_env(env: abi.dr_env_config, grids: TrackGrids, seed: int, true_theta: int) -> bytes:
    """The environment header as python-src/protocol.py packs a StratRaceEnvironmentConfig."""
    w = Writer()
    w.int32(MSG_HEADER)
    w.int32(ENV_STRATRACE)
    w.int32(1)
    w.array([env.n_theta])
    w.array(list(env.arena_min))
    w.array(list(env.arena_max))
    na = env.n_opp + 1
    w.int32(env.n_opp)
    w.int32(abi.DR_DIM)
    w.float32(env.dt)
    w.int32(env.send_states)
    for v in (env.drone_radius, env.pos_noise_level, env.speed_noise_level, env.action_noise_level):
        w.float32(v)
    w.array(list(env.max_speed)[:na])
    w.array(list(env.max_accel)[:na])
    w.int32(abi.DR_N_TRACK_SAMPLES)
    w.float32(env.track_width)
    w.int32(env.n_win_laps)
    w.int32(seed)
    w.array(list(env.init_belief)[: env.n_theta])
    for th in range(env.n_theta):
        oc = env.opp_configs[th]
        for name in ("s1", "s2", "s3", "speed_scale", "action_noise"):
            w.array(list(getattr(oc, name))[: env.n_opp])
    w.int32(true_theta)
    w.float32(env.kP)
    w.float32(env.kV)
    w.float32(env.max_opp_lat_dist_fact)
    w.float32(env.track_length)
    w.array(grids.p_grid)
    w.array(grids.dp_grid)
    w.array(grids.t_grid)
    w.array(grids.kappa_grid)
    return w.bytes()


def unpack_controller(buf: bytes) -> abi.dr_mppi_config | abi.dr_prmppi_config:
    """loadControllerConfig (src/config.cpp:86-115) and MPPIConfig / PRMPPIConfig
    ::unpackHeader (config.cpp:5-84)."""
    r = Reader(buf)
    if (k := r.int32()) != MSG_HEADER:
        raise ProtocolError(f"Expected header message type for controller config (type {MSG_HEADER}) but got type {k} instead")
    kind = r.int32()
    if kind == CONT_MPPI:
        c = abi.dr_mppi_config()
        c.n_samples = r.int32()
        c.n_timesteps = r.int32()
        c.n_knots = r.int32()
        if c.n_knots > abi.DR_MAX_KNOTS:
            raise ProtocolError(f"Received invalid number of knots: got {c.n_knots}, but at most {abi.DR_MAX_KNOTS} are supported")
        kn = r.array(at_most=abi.DR_MAX_KNOTS)
        if kn.size != c.n_knots:
            raise ProtocolError(f"Received invalid number of knots: got {kn.size} elements, but received nKnots={c.n_knots}")
        for i, v in enumerate(kn):
            c.knots[i] = int(v)
        c.use_splines = r.int32()
        # config.cpp:252-253 sets nKnots = nTimesteps in dense mode; the library does the
        # same internally, so the wire values are kept here (they re-encode identically)
        for name in ("inv_temperature", "sampling_noise", "gate_traversal_margin", "coll_dist_factor", "boundary_cost", "boundary_threshold_factor",
                     "outside_cost", "win_cost", "opp_win_cost", "final_adv_weight", "final_opp_adv_weight", "min_confidence"):
            setattr(c, name, r.float32())
        c.n_verif_samples = r.int32()
        c.beta = r.float32()
        c.verif_horizon = r.int32()
        c.max_verif_eps = r.float32()
        c.min_nu, c.max_nu, c.verify = 0.0005, 0.001, 1
        r.finished()
        return c
    if kind == CONT_PRMPPI:
        c = abi.dr_prmppi_config()
        c.n_samples = r.int32()
        c.n_timesteps = r.int32()
        for name in ("inv_temperature", "sampling_noise", "gate_traversal_margin", "coll_dist_factor", "boundary_cost", "boundary_threshold_factor",
                     "win_cost", "opp_win_cost", "final_adv_weight", "final_opp_adv_weight", "safety_weight", "min_safe_dist", "delta"):
            setattr(c, name, r.float32())
        c.P = r.int32()
        c.min_nu, c.max_nu = 0.0005, 0.001
        r.finished()
        return c
    raise ProtocolError(f"Received invalid controller kind {kind}")


def pack_controller(c) -> bytes:
    w = Writer()
    w.int32(MSG_HEADER)
    if isinstance(c, abi.dr_mppi_config):
        w.int32(CONT_MPPI)
        w.int32(c.n_samples)
        w.int32(c.n_timesteps)
        w.int32(c.n_knots if c.use_splines else c.n_knots)
        w.array(list(c.knots)[: c.n_knots])
        w.int32(c.use_splines)
        for name in ("inv_temperature", "sampling_noise", "gate_traversal_margin", "coll_dist_factor", "boundary_cost", "boundary_threshold_factor",
                     "outside_cost", "win_cost", "opp_win_cost", "final_adv_weight", "final_opp_adv_weight", "min_confidence"):
            w.float32(getattr(c, name))
        w.int32(c.n_verif_samples)
        w.float32(c.beta)
        w.int32(c.verif_horizon)
        w.float32(c.max_verif_eps)
    else:
        w.int32(CONT_PRMPPI)
        w.int32(c.n_samples)
        w.int32(c.n_timesteps)
        for name in ("inv_temperature", "sampling_noise", "gate_traversal_margin", "coll_dist_factor", "boundary_cost", "boundary_threshold_factor",
                     "win_cost", "opp_win_cost", "final_adv_weight", "final_opp_adv_weight", "safety_weight", "min_safe_dist", "delta"):
            w.float32(getattr(c, name))
        w.int32(c.P)
    return w.bytes()


def unpack_state(buf: bytes, n_opp: int) -> abi.dr_sim_state:
    """Env::unpackSimState (env_stratrace.cpp:98-118)."""
    r = Reader(buf)
    if (k := r.int32()) != MSG_HEADER:
        raise ProtocolError(f"Expected header message type for the initial state (type {MSG_HEADER}) but got type {k} instead")
    na = n_opp + 1
    s = abi.dr_sim_state()
    pos, vel, S, lat, laps = r.array(2 * na), r.array(2 * na), r.array(na), r.array(na), r.array(na)
    r.finished()
    for i in range(2 * na):
        s.pos[i] = float(pos[i])
        s.vel[i] = float(vel[i])
    for a in range(na):
        s.S[a] = float(S[a])
        s.lat_dist[a] = float(lat[a])
        s.laps[a] = int(laps[a])
    return s


def pack_state(s: abi.dr_sim_state, n_opp: int) -> bytes:
    na = n_opp + 1
    w = Writer()
    w.int32(MSG_HEADER)
    w.array(list(s.pos)[: 2 * na])
    w.array(list(s.vel)[: 2 * na])
    w.array(list(s.S)[:na])
    w.array(list(s.lat_dist)[:na])
    w.array(list(s.laps)[:na])
    return w.bytes()


def split_frames(blob: bytes) -> list[bytes]:
    """Frames stored as (uint32 length, bytes) records."""
    out, off = [], 0
    while off < len(blob):
        n = int.from_bytes(blob[off : off + 4], "little")
        out.append(blob[off + 4 : off + 4 + n])
        off += 4 + n
    return out


# ---- gate race (the reference's EnvDroneRace) -----------------------------------------

@dataclass
class GateEnvHeader:
    env: abi.dr_gate_env_config
    track: np.ndarray  # (DR_GATE_RACELINES, 512, 2) float32, referenced by env.track_points
    seed: int
    true_theta: int
    model_sizes: list[int]


def unpack_gate_env(buf: bytes) -> GateEnvHeader:
    """EnvDroneRace::unpackEnvConfig (env_dronerace.cpp:124-250), with this build's limits
    (2 agents, 2 racelines, up to 16 gates and 4 obstacles of each kind) in place of the
    reference's compile-time sizes."""
    r = Reader(buf)
    if (k := r.int32()) != MSG_HEADER:
        raise ProtocolError(f"Expected header message type for environment config (type {MSG_HEADER}) but got type {k} instead")
    if (ek := r.int32()) != ENV_DRONERACE:
        raise ProtocolError(f"Environment kind mismatch: received kind {ek}, but this decoder reads ENV_DRONERACE ({ENV_DRONERACE})")
    n_factors = r.int32()
    if n_factors != 1:
        raise ProtocolError(f"Received config for {n_factors} environment parameters but this build supports one parameter factor")
    sizes = [int(x) for x in r.array()]
    n_theta = sizes[0] if sizes else 0
    if not 1 <= n_theta <= abi.DR_MAX_THETA:
        raise ProtocolError(f"Received invalid model size {n_theta} (supported: 1..{abi.DR_MAX_THETA})")
    e = abi.dr_gate_env_config()
    e.n_theta = n_theta
    amin, amax = r.array(2), r.array(2)
    n_agents, dim = r.int32(), r.int32()
    e.dt = r.float32()
    e.send_states = r.int32()
    n_race, n_gates = r.int32(), r.int32()
    if n_agents != abi.DR_GATE_AGENTS:
        raise ProtocolError(f"Received config for {n_agents} agents but N_AGENTS is {abi.DR_GATE_AGENTS}")
    if dim != abi.DR_DIM:
        raise ProtocolError(f"Received config for dimension {dim} but DIM is {abi.DR_DIM}")
    if n_race != abi.DR_GATE_RACELINES:
        raise ProtocolError(f"Received config for {n_race} racelines but N_RACELINES is {abi.DR_GATE_RACELINES}")
    if not 1 <= n_gates <= abi.DR_GATE_MAX_GATES:
        raise ProtocolError(f"Received config for {n_gates} gates (supported: 1..{abi.DR_GATE_MAX_GATES})")
    for d in range(2):
        e.arena_min[d] = float(amin[d])
        e.arena_max[d] = float(amax[d])
    e.drone_radius = r.float32()
    e.pos_noise_level = r.float32()
    e.speed_noise_level = r.float32()
    e.action_noise_level = r.float32()
    ms, ma = r.array(2), r.array(2)
    for a in range(2):
        e.max_speed[a] = float(ms[a])
        e.max_accel[a] = float(ma[a])
    nts = r.int32()
    if nts != abi.DR_N_TRACK_SAMPLES:
        raise ProtocolError(f"Received config for {nts} track samples but N_TRACK_SAMPLES is {abi.DR_N_TRACK_SAMPLES}")
    e.n_win_laps = r.int32()
    e.target_distance = r.float32()
    e.n_gates = n_gates
    gc, gv, gr = r.array(2 * n_gates), r.array(2 * n_gates), r.array(n_gates)
    for i in range(2 * n_gates):
        e.gate_centers[i] = float(gc[i])
        e.gate_vectors[i] = float(gv[i])
    for i in range(n_gates):
        e.gate_radius[i] = float(gr[i])
    n_obs = r.int32()
    if not 0 <= n_obs <= abi.DR_GATE_MAX_OBSTACLES:
        raise ProtocolError(f"Received config for {n_obs} rect obstacles (supported: 0..{abi.DR_GATE_MAX_OBSTACLES})")
    obs = r.array(4 * n_obs)
    e.n_obstacles = n_obs
    for i in range(4 * n_obs):
        e.obstacles[i] = float(obs[i])
    n_round = r.int32()
    if not 0 <= n_round <= abi.DR_GATE_MAX_OBSTACLES:
        raise ProtocolError(f"Received config for {n_round} round obstacles (supported: 0..{abi.DR_GATE_MAX_OBSTACLES})")
    rc, rr = r.array(2 * n_round), r.array(n_round)
    e.n_round_obstacles = n_round
    for i in range(2 * n_round):
        e.round_obs_centers[i] = float(rc[i])
    for i in range(n_round):
        e.round_obs_radius[i] = float(rr[i])
    seed = r.int32()
    ib = r.array(n_theta)
    for th in range(n_theta):
        e.init_belief[th] = float(ib[th])
    for th in range(n_theta):  # unpackPIDConfig, env_dronerace.cpp:104-121
        p = e.opp_pid[th]
        p.kp, p.kd = r.float32(), r.float32()
        p.repulsion_factor, p.repulsion_power, p.repulsion_dist_fact = r.float32(), r.float32(), r.float32()
        p.raceline_index = r.int32()
        p.action_noise = r.float32()
    e.i_mppi = r.int32()
    true_theta = r.int32()
    tp = r.array(abi.DR_GATE_RACELINES * nts * 2)
    r.finished()
    track = np.ascontiguousarray(tp.reshape(abi.DR_GATE_RACELINES, nts, 2), np.float32)
    e.track_points = abi.fptr(track)
    return GateEnvHeader(e, track, seed, true_theta, sizes)


def pack_gate_env(env: abi.dr_gate_env_config, track: np.ndarray, seed: int, true_theta: int) -> bytes:
    """The environment header as python-src/protocol.py packs a DroneRaceEnvironmentConfig."""
    w = Writer()
    w.int32(MSG_HEADER)
    w.int32(ENV_DRONERACE)
    w.int32(1)
    w.array([env.n_theta])
    w.array(list(env.arena_min))
    w.array(list(env.arena_max))
    w.int32(abi.DR_GATE_AGENTS)
    w.int32(abi.DR_DIM)
    w.float32(env.dt)
    w.int32(env.send_states)
    w.int32(abi.DR_GATE_RACELINES)
    w.int32(env.n_gates)
    for v in (env.drone_radius, env.pos_noise_level, env.speed_noise_level, env.action_noise_level):
        w.float32(v)
    w.array(list(env.max_speed))
    w.array(list(env.max_accel))
    w.int32(abi.DR_N_TRACK_SAMPLES)
    w.int32(env.n_win_laps)
    w.float32(env.target_distance)
    ng = env.n_gates
    w.array(list(env.gate_centers)[: 2 * ng])
    w.array(list(env.gate_vectors)[: 2 * ng])
    w.array(list(env.gate_radius)[:ng])
    w.int32(env.n_obstacles)
    w.array(list(env.obstacles)[: 4 * env.n_obstacles])
    w.int32(env.n_round_obstacles)
    w.array(list(env.round_obs_centers)[: 2 * env.n_round_obstacles])
    w.array(list(env.round_obs_radius)[: env.n_round_obstacles])
    w.int32(seed)
    w.array(list(env.init_belief)[: env.n_theta])
    for th in range(env.n_theta):
        p = env.opp_pid[th]
        for v in (p.kp, p.kd, p.repulsion_factor, p.repulsion_power, p.repulsion_dist_fact):
            w.float32(v)
        w.int32(p.raceline_index)
        w.float32(p.action_noise)
    w.int32(env.i_mppi)
    w.int32(true_theta)
    w.array(np.asarray(track, np.float32).ravel())
    return w.bytes()


def unpack_gate_state(buf: bytes, i_mppi: int) -> abi.dr_gate_state:
    """EnvDroneRace::unpackSimState (env_dronerace.cpp:78-100): the ego's arc lengths are
    reset to -1 (untracked)."""
    r = Reader(buf)
    if (k := r.int32()) != MSG_HEADER:
        raise ProtocolError(f"Expected header message type for environment config (type {MSG_HEADER}) but got type {k} instead")
    na, nr = abi.DR_GATE_AGENTS, abi.DR_GATE_RACELINES
    pos, vel, S, laps, gates = r.array(2 * na), r.array(2 * na), r.array(na * nr), r.array(na), r.array(na)
    r.finished()
    s = abi.dr_gate_state()
    for i in range(2 * na):
        s.pos[i] = float(pos[i])
        s.vel[i] = float(vel[i])
    for i in range(na * nr):
        s.S[i] = float(S[i])
    for a in range(na):
        s.laps[a] = int(laps[a])
        s.gates[a] = int(gates[a])
    for k in range(nr):
        s.S[i_mppi * nr + k] = -1.0
    return s


def pack_gate_state(s: abi.dr_gate_state) -> bytes:
    w = Writer()
    w.int32(MSG_HEADER)
    w.array(list(s.pos))
    w.array(list(s.vel))
    w.array(list(s.S))
    w.array(list(s.laps))
    w.array(list(s.gates))
    return w.bytes()
