"""Track preprocessing on the device (track_kernels.cu, dr_track_grids) against the
restatement of the reference's front-end (track.track_grids: python-src/utils.py:390-427
with scipy's periodic CubicSpline), for the round track, seeded ellipses and seeded
jittered circles, many tracks in one launch."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import drb

pytestmark = pytest.mark.gpu

T = drb.track


def _tracks():
    fs = [T.circle_track(6.0), T.circle_track(20.0)]
    fs += [T.catmull_rom_closed(T.ellipse_points(s)) for s in range(4)]
    fs += [T.catmull_rom_closed(T.jittered_circle_points(s, 12)) for s in range(10)]
    return fs


def test_track_grids_on_device_match_reference_preprocessing(gpu):
    fs = _tracks()
    gpu_grids = T.track_grids_gpu(fs)
    exact = {"p": [], "t": []}
    for f, g in zip(fs, gpu_grids):
        c = T.track_grids(f)
        assert abs(g.track_length - c.track_length) <= 1e-6 * c.track_length
        for name in ("p_grid", "dp_grid", "t_grid"):
            np.testing.assert_allclose(getattr(g, name), getattr(c, name), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(g.kappa_grid, c.kappa_grid, rtol=1e-5, atol=1e-6)
        exact["p"].append(np.mean(g.p_grid == c.p_grid))
        exact["t"].append(np.mean(g.t_grid == c.t_grid))
    print({k: float(np.mean(v)) for k, v in exact.items()})
    # double precision on both sides: the float32 grids agree bit for bit almost everywhere
    assert np.mean(exact["p"]) > 0.99 and np.mean(exact["t"]) > 0.99
