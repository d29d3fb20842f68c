"""The certificate of the fast projection's local search (dr_projection_certificate, host
code, no GPU), checked by brute force in float64 on the float32 samples: at a point within
the certified radius of sample c where c is a local minimum of the squared distances
(to within the search's 1e-3 m^2 tolerance), every other sample of any window holding c is
farther by more than 1e-3 m^2. Tracks: the benchmark's jittered circles, ellipses, a small
circle and a hairpin (legs 1.5 m apart), where the certificate must shrink."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import drb

abi = drb.abi
T = drb.track
WIN = 10
EPS = 1e-3


def hairpin():
    return T.catmull_rom_closed(np.array([[0, 0], [10, 0], [20, 0], [21, 0.75], [20, 1.5], [10, 1.5], [0, 1.5], [-1, 0.75]], np.float64))


TRACKS = {
    "circle_r20": T.circle_track(20.0),
    "circle_r6": T.circle_track(6.0),
    "jittered_s0": T.catmull_rom_closed(T.jittered_circle_points(0, 12)),
    "jittered6_s3": T.catmull_rom_closed(T.jittered_circle_points(3, 6)),
    "ellipse_s1": T.catmull_rom_closed(T.ellipse_points(1)),
    "hairpin": hairpin(),
}


def certificate(p_grid: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(p_grid, np.float32)
    out = np.zeros(512, np.float32)
    abi.check(abi.lib().dr_projection_certificate(abi.fptr(p), abi.fptr(out)), "dr_projection_certificate")
    return out


def _lines():
    """(points [512][2], unit tangents [512][2]) of every track: the centrelines above and the
    gate race's racelines (ellipse offsets, the raceline walk's samples)."""
    out = {}
    for name, f in TRACKS.items():
        g = T.track_grids(f)
        out[name] = (g.p_grid, g.t_grid)
    for r, line in enumerate(drb.scenarios.ellipse_racelines()):
        d = np.roll(line, -1, axis=0) - np.roll(line, 1, axis=0)
        out[f"gate_raceline{r}"] = (np.ascontiguousarray(line, np.float32), (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32))
    return out


LINES = _lines()


@pytest.mark.parametrize("name", list(LINES))
def test_certificate_holds_by_brute_force(name):
    p_grid, t_grid = LINES[name]
    cert = certificate(p_grid)
    q = p_grid.astype(np.float64)
    rng = np.random.default_rng(7)
    checked = 0
    for c in range(512):
        if cert[c] <= 0:
            continue
        r = np.sqrt(cert[c])
        # points of the certified disk near the slab where c can be a local minimum:
        # along-track offsets within a sample spacing, lateral offsets across the disk
        t = t_grid[c].astype(np.float64)
        n = np.array([-t[1], t[0]])
        h = np.linalg.norm(q[(c + 1) % 512] - q[c])
        a = rng.uniform(-0.7 * h, 0.7 * h, 400)
        lat = rng.uniform(-r, r, 400)
        x = q[c] + a[:, None] * t + lat[:, None] * n
        x = x[((x - q[c]) ** 2).sum(axis=1) <= cert[c]]
        ks = (c + np.arange(-2 * WIN, 2 * WIN + 1)) % 512
        f = ((x[:, None, :] - q[ks][None, :, :]) ** 2).sum(axis=2)  # (points, 41)
        fc = f[:, 2 * WIN]
        local = (f[:, 2 * WIN - 1] - fc >= -EPS) & (f[:, 2 * WIN + 1] - fc >= -EPS)
        if not local.any():
            continue
        far = np.delete(f[local], [2 * WIN - 1, 2 * WIN, 2 * WIN + 1], axis=1)
        margin = far.min(axis=1) - fc[local]
        assert margin.min() > EPS, (name, c, float(margin.min()))
        checked += int(local.sum())
    assert checked > 10_000


def test_certificate_covers_the_track_band_and_shrinks_at_a_hairpin():
    """On the circles the certified radius is the 4 m cap everywhere; on the benchmark's
    track (12 points jittered around a circle, seed 0) it covers the whole track (half-width
    2 m, so every point still on the track certifies); at the hairpin's turns, where a window
    sees both legs, it drops below a metre (the kernel then scans the window)."""
    for name in ("circle_r20", "circle_r6", "jittered6_s3"):
        cert = certificate(T.track_grids(TRACKS[name]).p_grid)
        assert np.sqrt(cert.min()) > 3.99, name
    assert np.sqrt(certificate(T.track_grids(TRACKS["jittered_s0"]).p_grid).min()) > 2.1
    cert = certificate(T.track_grids(TRACKS["hairpin"]).p_grid)
    assert np.sqrt(np.clip(cert, 0, None)).min() < 1.0


def test_certificate_rejects_bad_input():
    bad = np.zeros((512, 2), np.float32)
    bad[3, 0] = np.nan
    out = np.zeros(512, np.float32)
    assert abi.lib().dr_projection_certificate(abi.fptr(bad), abi.fptr(out)) == abi.DR_ERR_INVALID_ARG
    # coincident samples certify nothing
    same = np.zeros((512, 2), np.float32)
    assert (certificate(same) < 0).all()
