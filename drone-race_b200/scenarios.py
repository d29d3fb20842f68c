"""Configuration builders: the reference's StratRace preset and the seeded synthetic
workloads the benchmark is quoted on.

`opp_preset` restates OppConfig.preset (python-src/utils.py:290-343); `strat_race`
restates stratRaceEnv (python-src/main.py:864-1000) with its MPPI / PR-MPPI settings.
The synthetic workloads map the benchmark's drone-race wording onto the reference's
2-D StratRace model (one ego agent plus policy opponents, a closed track of given
width, a discrete set of opponent hypotheses):
  * ellipse_race   1 agent, K=1024, H=50, dt=0.02, sigma=2.0, lambda=1.0, track through
                   8 control points on a 30 x 20 m ellipse, ego 3 m of arc behind the start;
  * circle_race    per agent: K=4096, H=64, dt=0.02, dense controls, track through 12
                   control points jittered +-5 m around a 40 m circle, drone radius 0.5,
                   collision weight 1e3;
  * robust_race    PR-MPPI, 8 opponent hypotheses (speed scale U(0.8,1.2), lateral
                   aggressiveness s1 U(0,2) m), belief ~ Dirichlet(1), P=8, K=2048, H=64.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .track import TrackGrids, catmull_rom_closed, circle_track, ellipse_points, jittered_circle_points, track_grids


def opp_preset(drone_radius: float, s1="default", s2="default", s3="default", speed_scale: float = 1.0, action_noise: float = 0.1) -> dict:
    """OppConfig.preset (python-src/utils.py:290-343) for one opponent."""
    r = drone_radius
    s1v = {"insensitive": 0.0, "default": 2.5 * r, "conservative": 4 * r}.get(s1, s1) if isinstance(s1, str) else s1
    s2v = {"infinite": 0.0, "default": 1 / (4 * r) ** 2, "insensitive": 1 / (1e-5 * r) ** 2}.get(s2, s2) if isinstance(s2, str) else s2
    s3v = {"no-block": 0.0, "default": 20 / r}.get(s3, s3) if isinstance(s3, str) else s3
    return dict(s1=float(s1v), s2=float(s2v), s3=float(s3v), speed_scale=float(speed_scale), action_noise=float(action_noise))


@dataclass
class Scenario:
    """Holds a C-ABI environment config together with the arrays its pointers refer to."""

    env: abi.dr_env_config
    grids: TrackGrids
    state: abi.dr_sim_state
    mppi: abi.dr_mppi_config | None = None
    prmppi: abi.dr_prmppi_config | None = None
    true_theta: int = 0
    seed: int = 42
    name: str = ""
    keep: list = field(default_factory=list)
    # controller kind in a mixed batch: "plain" MPPI, "grad" (gradient-refined MPPI) or "pr"
    kind: str = "plain"

    @property
    def n_theta(self) -> int:
        return int(self.env.n_theta)

    def belief(self) -> np.ndarray:
        return np.array(self.env.init_belief[: self.n_theta], dtype=np.float32)


def make_env(grids: TrackGrids, *, n_opp: int, opp_configs: list[list[dict]], dt: float, drone_radius: float, max_speed, max_accel,
             track_width: float, n_win_laps: int = 1, init_belief=None, kP: float = 10.0, kV: float = -1.0, max_opp_lat_dist_fact: float = 1.1,
             pos_noise: float = 0.0, speed_noise: float = 0.0, action_noise: float = 0.0) -> abi.dr_env_config:
    """EnvironmentConfig (env_stratrace_defs.h:53-86); opp_configs[theta][opp]."""
    e = abi.dr_env_config()
    n_theta = len(opp_configs)
    e.n_opp = n_opp
    e.n_theta = n_theta
    pmin = grids.p_grid.min(axis=0) - track_width * 2  # utils.py:429-431
    pmax = grids.p_grid.max(axis=0) + track_width * 2
    for d in range(2):
        e.arena_min[d] = float(pmin[d])
        e.arena_max[d] = float(pmax[d])
    e.dt = dt
    e.send_states = 1
    e.drone_radius = drone_radius
    e.pos_noise_level = pos_noise
    e.speed_noise_level = speed_noise
    e.action_noise_level = action_noise
    for a in range(n_opp + 1):
        e.max_speed[a] = float(max_speed[a])
        e.max_accel[a] = float(max_accel[a])
    e.track_width = track_width
    e.n_win_laps = n_win_laps
    if init_belief is None:
        init_belief = np.full(n_theta, 1.0 / n_theta)
    for th in range(n_theta):
        e.init_belief[th] = float(np.float32(init_belief[th]))
        for o in range(n_opp):
            oc = opp_configs[th][o]
            e.opp_configs[th].s1[o] = oc["s1"]
            e.opp_configs[th].s2[o] = oc["s2"]
            e.opp_configs[th].s3[o] = oc["s3"]
            e.opp_configs[th].speed_scale[o] = oc["speed_scale"]
            e.opp_configs[th].action_noise[o] = oc["action_noise"]
    e.kP = kP
    e.kV = 2 * kP**0.5 if kV == -1.0 else kV  # utils.py:387-388
    e.max_opp_lat_dist_fact = max_opp_lat_dist_fact
    e.track_length = grids.track_length
    e.p_grid = abi.fptr(grids.p_grid)
    e.dp_grid = abi.fptr(grids.dp_grid)
    e.t_grid = abi.fptr(grids.t_grid)
    e.kappa_grid = abi.fptr(grids.kappa_grid)
    return e


def initial_state(grids: TrackGrids, sample_idx: list[int], n_opp: int) -> abi.dr_sim_state:
    """Agents at rest on the centreline at the given track samples (main.py:908-916)."""
    s = abi.dr_sim_state()
    for a in range(n_opp + 1):
        i = int(sample_idx[a]) % 512
        s.pos[2 * a] = float(grids.p_grid[i, 0])
        s.pos[2 * a + 1] = float(grids.p_grid[i, 1])
        s.S[a] = float(np.float32(i / 512 * grids.track_length))
    return s


def default_knots(T: int, M: int) -> np.ndarray:
    """MPPIConfig.__post_init__ default knots (utils.py:496-498): tau_(M-1) <= T-2."""
    return np.arange(0, M) * int((T - 2) / (M - 1))


def make_mppi(*, K: int, T: int, use_splines: bool, M: int = 20, knots=None, inv_temperature=10.0, sampling_noise=0.5, coll_dist_factor=1.4,
              boundary_cost=50.0, boundary_threshold_factor=1.8, outside_cost=1e7, win_cost=1e5, opp_win_cost=1e5, final_adv_weight=50.0,
              final_opp_adv_weight=0.0, min_confidence=0.95, n_verif_samples=2**17, beta=1e-5, verif_horizon=40, max_verif_eps=0.001,
              gate_traversal_margin=0.95, verify=True) -> abi.dr_mppi_config:
    """MPPIConfig (include/config.h:116-154); defaults are stratRaceEnv's spline MPPI
    (main.py:945-968) with the verification settings of main.py:1021-1025."""
    c = abi.dr_mppi_config()
    c.n_samples = K
    c.n_timesteps = T
    if use_splines:
        c.n_knots = M
        kn = default_knots(T, M) if knots is None else np.asarray(knots)
        for i, v in enumerate(kn):
            c.knots[i] = int(v)
    else:
        c.n_knots = T
        for i in range(min(T, abi.DR_MAX_KNOTS)):
            c.knots[i] = i
    c.use_splines = int(bool(use_splines))
    c.inv_temperature = inv_temperature
    c.sampling_noise = sampling_noise
    c.gate_traversal_margin = gate_traversal_margin
    c.coll_dist_factor = coll_dist_factor
    c.boundary_cost = boundary_cost
    c.boundary_threshold_factor = boundary_threshold_factor
    c.outside_cost = outside_cost
    c.win_cost = win_cost
    c.opp_win_cost = opp_win_cost
    c.final_adv_weight = final_adv_weight
    c.final_opp_adv_weight = final_opp_adv_weight
    c.min_confidence = min_confidence
    c.n_verif_samples = n_verif_samples
    c.beta = beta
    c.verif_horizon = min(verif_horizon, T)
    c.max_verif_eps = max_verif_eps
    c.sampling_noise_dim[0] = 0.0
    c.sampling_noise_dim[1] = 0.0
    c.min_nu = 0.0005
    c.max_nu = 0.001
    c.verify = int(bool(verify))
    return c


def make_prmppi(*, K: int, T: int, P: int = 0, delta: float = 0.1, inv_temperature=10.0, sampling_noise=0.5, coll_dist_factor=1.2, boundary_cost=20.0,
                boundary_threshold_factor=1.3, win_cost=1e6, opp_win_cost=1e5, final_adv_weight=500.0, final_opp_adv_weight=0.0, safety_weight=1e4,
                min_safe_dist=0.0, gate_traversal_margin=0.9) -> abi.dr_prmppi_config:
    """PRMPPIConfig (include/config.h:157-192); defaults are stratRaceEnv's PR-MPPI
    (main.py:971-993); P = ceil((1-delta)/delta) when not given (utils.py:537-538)."""
    import math

    c = abi.dr_prmppi_config()
    c.n_samples = K
    c.n_timesteps = T
    c.inv_temperature = inv_temperature
    c.sampling_noise = sampling_noise
    c.gate_traversal_margin = gate_traversal_margin
    c.coll_dist_factor = coll_dist_factor
    c.boundary_cost = boundary_cost
    c.boundary_threshold_factor = boundary_threshold_factor
    c.win_cost = win_cost
    c.opp_win_cost = opp_win_cost
    c.final_adv_weight = final_adv_weight
    c.final_opp_adv_weight = final_opp_adv_weight
    c.safety_weight = safety_weight
    c.min_safe_dist = min_safe_dist
    c.delta = delta
    c.P = P if P else math.ceil((1 - delta) / delta)
    c.min_nu = 0.0005
    c.max_nu = 0.001
    return c


def strat_race(use_pr: bool = False, use_splines: bool = True, n_configs: int = 2, first_config: int = 0, K: int | None = None,
               T: int | None = None, action_noise: float = 0.1, n_verif: int = 2**17) -> Scenario:
    """stratRaceEnv (python-src/main.py:864-1000) with mppiPos = 0."""
    r = 0.4
    presets = [
        opp_preset(r, s1="insensitive", s3="default", action_noise=action_noise),
        opp_preset(r, s1="insensitive", s3="no-block", action_noise=action_noise),
        opp_preset(r, s1="default", s3="default", action_noise=action_noise),
        opp_preset(r, s1="conservative", s3="no-block", action_noise=action_noise),
    ][first_config : first_config + n_configs]
    grids = track_grids(circle_track(6.0))
    env = make_env(grids, n_opp=1, opp_configs=[[p] for p in presets], dt=0.1, drone_radius=r, max_speed=[3, 2], max_accel=[2, 3], track_width=2.0,
                   kV=5.0, max_opp_lat_dist_fact=1.9)
    init_idx = np.round(np.linspace(0.05, 0.2, 2) * 512).astype(int)
    st = initial_state(grids, list(init_idx), 1)
    sc = Scenario(env=env, grids=grids, state=st, name="strat_race")
    if use_pr:
        sc.prmppi = make_prmppi(K=K or 2**16, T=T or 60)
    elif use_splines:
        TT = T or 80
        sc.mppi = make_mppi(K=K or 2**16, T=TT, use_splines=True, M=min(20, max(2, (TT - 2) // 2)), n_verif_samples=n_verif)
    else:
        sc.mppi = make_mppi(K=K or 2**16, T=T or 70, use_splines=False, inv_temperature=10, sampling_noise=1.5, coll_dist_factor=1.3,
                            final_adv_weight=500, boundary_cost=50, boundary_threshold_factor=1.7, outside_cost=1e6, win_cost=1e6, opp_win_cost=1e5,
                            n_verif_samples=n_verif)
    return sc


def _start_indices(grids: TrackGrids, ego_offset_m: float, opp_gap_m: float, shift: int) -> list[int]:
    per = grids.track_length / 512
    ego = int(round(-ego_offset_m / per)) + shift
    opp = ego + int(round(opp_gap_m / per))
    return [ego % 512, opp % 512]


def ellipse_race(seed: int = 0, K: int = 1024, T: int = 50, use_splines: bool = False, n_verif: int = 4096) -> Scenario:
    """Single-agent MPPI on a track through 8 control points of a 30 x 20 m ellipse."""
    r = 0.4
    grids = track_grids(catmull_rom_closed(ellipse_points(seed, 8)))
    presets = [opp_preset(r, s1="insensitive", s3="default"), opp_preset(r, s1="insensitive", s3="no-block")]
    env = make_env(grids, n_opp=1, opp_configs=[[p] for p in presets], dt=0.02, drone_radius=r, max_speed=[6, 4], max_accel=[6, 6], track_width=1.5,
                   kV=5.0, max_opp_lat_dist_fact=1.9)
    st = initial_state(grids, _start_indices(grids, 3.0, 4.0, 0), 1)
    sc = Scenario(env=env, grids=grids, state=st, seed=seed, name="ellipse_race")
    sc.mppi = make_mppi(K=K, T=T, use_splines=use_splines, M=min(20, T // 2), inv_temperature=1.0, sampling_noise=2.0, n_verif_samples=n_verif,
                        verif_horizon=min(40, T), outside_cost=1e3)
    return sc


_CIRCLE_GRIDS: dict[tuple[int, int], TrackGrids] = {}


def _circle_grids(seed: int, n_points: int) -> TrackGrids:
    key = (seed, n_points)
    if key not in _CIRCLE_GRIDS:
        _CIRCLE_GRIDS[key] = track_grids(catmull_rom_closed(jittered_circle_points(seed, n_points)))
    return _CIRCLE_GRIDS[key]


def circle_race(agent: int = 0, seed: int = 0, K: int = 4096, T: int = 64, use_splines: bool = False, n_theta: int = 2, n_verif: int = 2**17,
                sampling_noise: float = 1.0, n_points: int = 12) -> Scenario:
    """Per-agent MPPI workload of the 4-agent benchmark: a closed Catmull-Rom track
    through n_points (12) control points jittered +-5 m around a 40 m circle (seeded),
    drone radius 0.5, collision (outside) weight 1e3, lambda = 1. Agents start at
    different places along the same track."""
    r = 0.5
    grids = _circle_grids(seed, n_points)
    base = [opp_preset(r, s1="insensitive", s3="default"), opp_preset(r, s1="insensitive", s3="no-block"),
            opp_preset(r, s1="default", s3="default"), opp_preset(r, s1="conservative", s3="no-block")]
    presets = [base[i % 4] for i in range(n_theta)]
    env = make_env(grids, n_opp=1, opp_configs=[[p] for p in presets], dt=0.02, drone_radius=r, max_speed=[6, 4], max_accel=[6, 6], track_width=2.0,
                   kV=5.0, max_opp_lat_dist_fact=1.9)
    st = initial_state(grids, _start_indices(grids, 3.0, 4.0, agent * 128), 1)
    sc = Scenario(env=env, grids=grids, state=st, seed=seed * 1000 + agent, name="circle_race")
    sc.mppi = make_mppi(K=K, T=T, use_splines=use_splines, M=20, inv_temperature=1.0, sampling_noise=sampling_noise, n_verif_samples=n_verif,
                        verif_horizon=min(40, T), outside_cost=1e3)
    return sc


def uneven_races(n_races: int = 256, seed: int = 0, n_verif: int = 4096) -> list[Scenario]:
    """Many independent races of uneven sizes, one scenario per agent: per race U{1..8}
    agents on a track through U{6..16} control points jittered around a 40 m circle, and
    one control mode (dense or spline controls, alternating by race); per agent K
    log-uniform in [256, 16384] and H in {32, 48, 64, 96}, verification of n_verif
    samples over min(40, H) steps. `Scenario.name` is "race<r>/agent<a>"."""
    rng = np.random.default_rng(50_000 + seed)
    out = []
    for race in range(n_races):
        n_agents = int(rng.integers(1, 9))
        n_points = int(rng.integers(6, 17))
        spl = bool(race % 2)
        for a in range(n_agents):
            K = int(round(float(np.exp(rng.uniform(np.log(256), np.log(16384))))))
            T = int(rng.choice([32, 48, 64, 96]))
            sc = circle_race(agent=a, seed=seed * 100_000 + race, K=K, T=T, use_splines=spl, n_verif=n_verif, n_points=n_points)
            sc.name = f"race{race}/agent{a}"
            out.append(sc)
    return out


def mixed_races(n_races: int = 256, seed: int = 0, n_verif: int = 4096) -> list[Scenario]:
    """The batched uneven workload of many independent races of mixed controller kinds, one
    scenario per agent: per race U{1..8} agents on a track through U{6..16} control points
    jittered around a 40 m circle and one kind (`Scenario.kind`): plain MPPI (about half the
    races, dense or spline controls alternating), gradient-refined MPPI (about a quarter: one
    projected gradient step after each update) or PR-MPPI with B in {2, 4, 8} belief
    branches (about a quarter: B opponent hypotheses under a Dirichlet(1) belief, P = B
    sampled hypotheses). Per agent K log-uniform in [256, 16384] and H in {32, 48, 64, 96};
    MPPI verification of n_verif samples over min(40, H) steps."""
    rng = np.random.default_rng(60_000 + seed)
    out = []
    for race in range(n_races):
        n_agents = int(rng.integers(1, 9))
        n_points = int(rng.integers(6, 17))
        u = float(rng.uniform())
        kind = "plain" if u < 0.5 else ("grad" if u < 0.75 else "pr")
        B = int(rng.choice([2, 4, 8]))
        spl = bool(race % 2)
        for a in range(n_agents):
            K = int(round(float(np.exp(rng.uniform(np.log(256), np.log(16384))))))
            T = int(rng.choice([32, 48, 64, 96]))
            if kind == "pr":
                sc = robust_race(agent=a, seed=seed * 100_000 + race, K=K, T=T, P=B, n_theta=B, n_points=n_points)
            else:
                sc = circle_race(agent=a, seed=seed * 100_000 + race, K=K, T=T, use_splines=spl, n_verif=n_verif, n_points=n_points)
            sc.kind = kind
            sc.name = f"race{race}/agent{a}"
            out.append(sc)
    return out


def robust_race(agent: int = 0, seed: int = 0, K: int = 2048, T: int = 64, P: int = 8, n_theta: int = 8, n_points: int = 12) -> Scenario:
    """Per-agent PR-MPPI workload: n_theta opponent hypotheses (speed scale U(0.8,1.2),
    lateral aggressiveness s1 U(0,2) m), belief ~ Dirichlet(1), P sampled hypotheses, on a
    track through n_points control points jittered around a 40 m circle."""
    r = 0.5
    rng = np.random.default_rng(10_000 + seed * 100 + agent)
    grids = _circle_grids(seed, n_points)
    presets = []
    for th in range(n_theta):
        presets.append(opp_preset(r, s1=float(rng.uniform(0, 2)), s3="default" if th % 2 == 0 else "no-block", speed_scale=float(rng.uniform(0.8, 1.2))))
    belief = rng.dirichlet(np.ones(n_theta)).astype(np.float32)
    belief = belief / belief.sum(dtype=np.float32)
    env = make_env(grids, n_opp=1, opp_configs=[[p] for p in presets], dt=0.02, drone_radius=r, max_speed=[6, 4], max_accel=[6, 6], track_width=2.0,
                   kV=5.0, max_opp_lat_dist_fact=1.9, init_belief=belief)
    st = initial_state(grids, _start_indices(grids, 3.0, 4.0, agent * 128), 1)
    sc = Scenario(env=env, grids=grids, state=st, seed=seed * 1000 + agent, name="robust_race")
    sc.prmppi = make_prmppi(K=K, T=T, P=P, inv_temperature=1.0, sampling_noise=1.0)
    return sc


# ==== gate race (the reference's EnvDroneRace) ==========================================

@dataclass
class GateScenario:
    """A gate-race environment (C-ABI struct) with the racelines it points to."""

    env: abi.dr_gate_env_config
    track: np.ndarray  # (DR_GATE_RACELINES, 512, 2) float32, referenced by env.track_points
    state: abi.dr_gate_state
    mppi: abi.dr_mppi_config | None = None
    true_theta: int = 0
    seed: int = 42
    name: str = ""

    @property
    def n_theta(self) -> int:
        return int(self.env.n_theta)

    def belief(self) -> np.ndarray:
        return np.array(self.env.init_belief[: self.n_theta], dtype=np.float32)


def pid_config(kp: float = 5.0, kd: float = 20.0, repulsion_factor: float = 0.0, repulsion_power: float = 2.0, repulsion_dist_fact: float = 10.0,
               raceline_index: int = 0, action_noise: float = 0.0) -> abi.dr_pid_config:
    """PIDConfig (env_dronerace_defs.h:44-56); defaults of python-src/main.py:65-66."""
    p = abi.dr_pid_config()
    p.kp, p.kd = kp, kd
    p.repulsion_factor, p.repulsion_power, p.repulsion_dist_fact = repulsion_factor, repulsion_power, repulsion_dist_fact
    p.raceline_index = raceline_index
    p.action_noise = action_noise
    return p


def ellipse_racelines(a: float = 15.0, b: float = 10.0, offsets=(-0.6, 0.6), n: int = abi.DR_N_TRACK_SAMPLES) -> np.ndarray:
    """Racelines parallel to an a x b ellipse (semi-axes), offset along its outward
    normal, sampled at n equal parameter steps counter-clockwise: (len(offsets), n, 2)."""
    u = np.arange(n) * (2 * np.pi / n)
    c = np.stack([a * np.cos(u), b * np.sin(u)], axis=1)
    t = np.stack([-a * np.sin(u), b * np.cos(u)], axis=1)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    nrm = np.stack([t[:, 1], -t[:, 0]], axis=1)  # outward for a counter-clockwise loop
    return np.stack([c + o * nrm for o in offsets]).astype(np.float32)


def ellipse_gates(n_gates: int, a: float = 15.0, b: float = 10.0, radius: float = 1.5, seed: int | None = None):
    """n_gates gates on an a x b ellipse, facing along the race direction (counter-
    clockwise), at equal parameter steps (uniform random angles, sorted, when seeded)."""
    if seed is None:
        u = np.arange(n_gates) * (2 * np.pi / n_gates)
    else:
        u = np.sort(np.random.default_rng(seed).uniform(0, 2 * np.pi, n_gates))
    centers = np.stack([a * np.cos(u), b * np.sin(u)], axis=1)
    vec = np.stack([-a * np.sin(u), b * np.cos(u)], axis=1)
    vec /= np.linalg.norm(vec, axis=1, keepdims=True)
    return centers.astype(np.float32), vec.astype(np.float32), np.full(n_gates, radius, np.float32)


def make_gate_env(track: np.ndarray, centers, vectors, radius, pids: list, *, dt: float, drone_radius: float, max_speed, max_accel,
                  target_distance: float = 0.05, n_win_laps: int = 1, init_belief=None, i_mppi: int = 0, arena_margin: float = 3.0,
                  pos_noise: float = 0.0, speed_noise: float = 0.0, action_noise: float = 0.0, round_obstacles=(), rect_obstacles=()) -> abi.dr_gate_env_config:
    """EnvironmentConfig of the gate race (env_dronerace_defs.h:60-93)."""
    e = abi.dr_gate_env_config()
    n_theta = len(pids)
    e.n_theta = n_theta
    lo = track.reshape(-1, 2).min(axis=0) - arena_margin
    hi = track.reshape(-1, 2).max(axis=0) + arena_margin
    for d in range(2):
        e.arena_min[d] = float(lo[d])
        e.arena_max[d] = float(hi[d])
    e.dt = dt
    e.send_states = 1
    e.drone_radius = drone_radius
    e.pos_noise_level, e.speed_noise_level, e.action_noise_level = pos_noise, speed_noise, action_noise
    for a in range(2):
        e.max_speed[a] = float(max_speed[a])
        e.max_accel[a] = float(max_accel[a])
    e.n_win_laps = n_win_laps
    e.target_distance = target_distance
    e.n_gates = len(centers)
    for g in range(len(centers)):
        for d in range(2):
            e.gate_centers[2 * g + d] = float(centers[g][d])
            e.gate_vectors[2 * g + d] = float(vectors[g][d])
        e.gate_radius[g] = float(radius[g])
    e.n_round_obstacles = len(round_obstacles)
    for i, (cx, cy, rr) in enumerate(round_obstacles):
        e.round_obs_centers[2 * i], e.round_obs_centers[2 * i + 1], e.round_obs_radius[i] = cx, cy, rr
    e.n_obstacles = len(rect_obstacles)
    for i, box in enumerate(rect_obstacles):
        for j in range(4):
            e.obstacles[4 * i + j] = float(box[j])
    e.track_points = abi.fptr(track)
    if init_belief is None:
        init_belief = np.full(n_theta, 1.0 / n_theta)
    for th in range(n_theta):
        e.init_belief[th] = float(np.float32(init_belief[th]))
        e.opp_pid[th] = pids[th]
    e.i_mppi = i_mppi
    return e


def gate_state(track: np.ndarray, start_u: list[float], i_mppi: int, gates: list[int], speed: float = 0.0) -> abi.dr_gate_state:
    """Both agents on raceline 0 at the given fractions of a lap, moving along it at
    `speed`; each opponent's S on every raceline is its fraction of a lap, the ego's is
    -1 (untracked, as env_dronerace.cpp:96-97 loads it)."""
    s = abi.dr_gate_state()
    n = track.shape[1]
    for a in range(2):
        i = int(round(start_u[a] * n)) % n
        p = track[0, i]
        q = track[0, (i + 1) % n] - track[0, i - 1]
        q = q / np.linalg.norm(q)
        s.pos[2 * a], s.pos[2 * a + 1] = float(p[0]), float(p[1])
        s.vel[2 * a], s.vel[2 * a + 1] = float(speed * q[0]), float(speed * q[1])
        for r in range(abi.DR_GATE_RACELINES):
            s.S[a * abi.DR_GATE_RACELINES + r] = -1.0 if a == i_mppi else float(np.float32(i / n))
        s.laps[a] = 0
        s.gates[a] = gates[a]
    return s


def gate_race(agent: int = 0, seed: int = 0, K: int = 4096, T: int = 64, use_splines: bool = False, n_verif: int = 2**17, n_gates: int = 2,
              action_noise: float = 0.5, i_mppi: int = 0) -> GateScenario:
    """Gate race on a 30 x 20 m ellipse: n_gates gates of radius 1.5 m facing the race
    direction, two racelines 0.6 m inside and outside the ellipse, one PID opponent whose
    hypotheses follow either raceline (kp 5, kd 20, python-src/main.py:65-66), drone
    radius 0.5, dt 0.02; the MPPI settings of tinyGateEnv (main.py:140-189). The agents
    start a metre or two apart just past a gate (the opponent ahead), so a lap is the
    whole loop; `agent` shifts the start around the loop."""
    track = ellipse_racelines()
    centers, vectors, radius = ellipse_gates(n_gates)
    pids = [pid_config(raceline_index=0, action_noise=action_noise), pid_config(raceline_index=1, action_noise=action_noise)]
    env = make_gate_env(track, centers, vectors, radius, pids, dt=0.02, drone_radius=0.5, max_speed=[6.0, 4.0], max_accel=[6.0, 6.0],
                        target_distance=0.05, i_mppi=i_mppi)
    shift = 0.37 * agent
    ego_u, opp_u = (0.01 + shift) % 1.0, (0.035 + shift) % 1.0
    # gates[a]: last gate passed; the next one is the first gate ahead of the start
    next_gate = int(np.searchsorted(np.arange(n_gates) / n_gates, (ego_u + 1e-9) % 1.0)) % n_gates
    last = (next_gate - 1) % n_gates
    start = [ego_u, opp_u] if i_mppi == 0 else [opp_u, ego_u]
    st = gate_state(track, start, i_mppi, [last, last], speed=2.0)
    sc = GateScenario(env=env, track=track, state=st, seed=seed * 1000 + agent, name="gate_race")
    sc.mppi = make_mppi(K=K, T=T, use_splines=use_splines, M=min(10, max(2, (T - 2) // 2)), inv_temperature=10.0, sampling_noise=2.0,
                        coll_dist_factor=1.1, final_adv_weight=200.0, boundary_cost=0.0, boundary_threshold_factor=1.7, outside_cost=1e6, win_cost=1e6,
                        opp_win_cost=1e5, n_verif_samples=n_verif, verif_horizon=min(40, T), gate_traversal_margin=0.9)
    return sc
