"""Track preprocessing and seeded synthetic tracks.

`track_grids` restates the StratRace track preprocessing of the reference's Python
front-end (python-src/utils.py:390-427): the closed curve given by a track function is
sampled at 512 points, re-parametrised by arc length with a periodic cubic spline, and
turned into the position / derivative / unit-tangent / curvature grids the model reads.

The synthetic generators make the seeded tracks the benchmark configurations are
quoted on (an ellipse through randomly placed control points, and a closed
Catmull-Rom spline through control points jittered around a circle).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np
from scipy.interpolate import CubicSpline

N_TRACK_SAMPLES = 512


@dataclass
class TrackGrids:
    track_length: float
    p_grid: np.ndarray  # (512, 2) float32
    dp_grid: np.ndarray  # (512, 2)
    t_grid: np.ndarray  # (512, 2) unit tangent
    kappa_grid: np.ndarray  # (512,) curvature


def track_grids(track_function: Callable[[float], np.ndarray], n: int = N_TRACK_SAMPLES) -> TrackGrids:
    """python-src/utils.py:391-427, computed in float64 and stored as float32 (the wire
    format sends float32, protocol.py:25-30)."""
    q = np.array([track_function(k / n) for k in range(n)], dtype=np.float64)
    diffs = np.diff(q, axis=0, append=q[0:1])
    d_k = np.linalg.norm(diffs, axis=1)
    s_k = np.zeros(n + 1)
    s_k[1:] = np.cumsum(d_k)
    L = s_k[-1]
    q_periodic = np.vstack([q, q[0:1]])
    cs_x = CubicSpline(s_k, q_periodic[:, 0], bc_type="periodic")
    cs_y = CubicSpline(s_k, q_periodic[:, 1], bc_type="periodic")
    s_grid = np.linspace(0, L, n, endpoint=False)
    p = np.column_stack([cs_x(s_grid), cs_y(s_grid)])
    dx, dy = cs_x(s_grid, 1), cs_y(s_grid, 1)
    dp = np.column_stack([dx, dy])
    dp_norm = np.linalg.norm(dp, axis=1, keepdims=True)
    t = dp / np.maximum(dp_norm, 1e-6)
    ddx, ddy = cs_x(s_grid, 2), cs_y(s_grid, 2)
    kappa = (dx * ddy - dy * ddx) / np.maximum((dx**2 + dy**2) ** 1.5, 1e-6)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return TrackGrids(float(np.float32(L)), f32(p), f32(dp), f32(t), f32(kappa))


def track_grids_gpu(track_functions: list[Callable[[float], np.ndarray]], n: int = N_TRACK_SAMPLES) -> list[TrackGrids]:
    """`track_grids` for many tracks at once on the GPU (dr_track_grids): the track
    functions are sampled here, the arc-length spline and the grids are computed on the
    device, one CTA per track."""
    import ctypes as C

    from . import abi

    if n != N_TRACK_SAMPLES:
        raise ValueError("the device path samples 512 points per track")
    R = len(track_functions)
    q = np.ascontiguousarray(np.stack([np.array([f(k / n) for k in range(n)], dtype=np.float64) for f in track_functions]))
    p = np.zeros((R, n, 2), np.float32)
    dp = np.zeros((R, n, 2), np.float32)
    t = np.zeros((R, n, 2), np.float32)
    kap = np.zeros((R, n), np.float32)
    L = np.zeros(R, np.float32)
    abi.check(abi.lib().dr_track_grids(q.ctypes.data_as(C.POINTER(C.c_double)), R, abi.fptr(p), abi.fptr(dp), abi.fptr(t), abi.fptr(kap), abi.fptr(L)),
              "dr_track_grids")
    return [TrackGrids(float(L[r]), p[r], dp[r], t[r], kap[r]) for r in range(R)]


def circle_track(radius: float = 6.0) -> Callable[[float], np.ndarray]:
    """The reference's round track (python-src/main.py:867-868)."""
    return lambda f: radius * np.array([np.cos(2 * np.pi * f), np.sin(2 * np.pi * f)])


def catmull_rom_closed(points: np.ndarray) -> Callable[[float], np.ndarray]:
    """Closed uniform Catmull-Rom curve through `points` (n, 2), parameter f in [0, 1)."""
    P = np.asarray(points, dtype=np.float64)
    n = len(P)

    def f(u: float) -> np.ndarray:
        x = (u % 1.0) * n
        i = int(np.floor(x)) % n
        t = x - np.floor(x)
        p0, p1, p2, p3 = P[(i - 1) % n], P[i], P[(i + 1) % n], P[(i + 2) % n]
        t2, t3 = t * t, t * t * t
        return 0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t2 + (-p0 + 3 * p1 - 3 * p2 + p3) * t3)

    return f


def ellipse_points(seed: int, n: int = 8, a: float = 15.0, b: float = 10.0) -> np.ndarray:
    """n control points on an a x b semi-axis ellipse (a 30 x 20 m ellipse) at sorted
    uniform-random angles."""
    rng = np.random.default_rng(seed)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    return np.column_stack([a * np.cos(ang), b * np.sin(ang)])


def jittered_circle_points(seed: int, n: int = 12, radius: float = 20.0, jitter: float = 5.0) -> np.ndarray:
    """n control points evenly spaced on a circle (40 m across), each jittered
    uniformly by +-jitter m in x and y."""
    rng = np.random.default_rng(seed)
    ang = np.arange(n) * 2 * np.pi / n
    base = np.column_stack([radius * np.cos(ang), radius * np.sin(ang)])
    return base + rng.uniform(-jitter, jitter, size=(n, 2))
