"""The projection onto the centreline: the certified local search of the window gives bit
for bit the arc length, lateral distance and sample of the full window scan, in the fast
flavour (dr_debug_project mode 0 against 1, what mppi_verify runs) and in the exact one
(mode 2 against 3: the rollout's search against the reference's scan as written), on
smooth tracks, on a hairpin whose windows see both legs, for points on and far off the
track and for previous arc lengths up to nine samples away (walks to the window's edge,
where the search hands over to the scan)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import drb
from test_projection_cert import TRACKS

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios
T = drb.track


def _env(grids):
    return S.make_env(grids, n_opp=1, opp_configs=[[S.opp_preset(0.5)]], dt=0.02, drone_radius=0.5, max_speed=[6, 4], max_accel=[6, 6],
                      track_width=2.0)


def _points(grids, n, seed):
    rng = np.random.default_rng(seed)
    L = grids.track_length
    q = grids.p_grid.astype(np.float64)
    t = grids.t_grid.astype(np.float64)
    c = rng.integers(0, 512, n)
    h = L / 512
    u = rng.uniform(size=n)
    lat = np.where(u < 0.8, rng.uniform(-2.5, 2.5, n), np.where(u < 0.95, rng.uniform(-6, 6, n), rng.uniform(-12, 12, n)))
    along = rng.uniform(-0.6, 0.6, n) * h
    nrm = np.column_stack([-t[c, 1], t[c, 0]])
    xy = q[c] + along[:, None] * t[c] + lat[:, None] * nrm
    shift = np.where(rng.uniform(size=n) < 0.9, rng.uniform(-3, 3, n), rng.uniform(-9, 9, n))
    prev = np.mod(c + shift, 512) * h
    return np.ascontiguousarray(xy, np.float32), np.ascontiguousarray(prev, np.float32)


def _project(env, xy, prev, mode):
    n = len(prev)
    s = np.zeros(n, np.float32)
    lat = np.zeros(n, np.float32)
    idx = np.zeros(n, np.int32)
    abi.check(abi.lib().dr_debug_project(env, abi.fptr(xy), abi.fptr(prev), n, mode, abi.fptr(s), abi.fptr(lat), abi.iptr(idx)), "dr_debug_project")
    return s, lat, idx


@pytest.mark.parametrize("name", list(TRACKS))
def test_local_search_equals_window_scan(gpu, name):
    grids = T.track_grids(TRACKS[name])
    env = _env(grids)
    xy, prev = _points(grids, 200_000, seed=list(TRACKS).index(name))
    a = _project(env, xy, prev, 0)
    b = _project(env, xy, prev, 1)
    for x, y in zip(a, b):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    e = _project(env, xy, prev, 2)
    for x, y in zip(e, _project(env, xy, prev, 3)):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    # the two flavours agree to within the fast flavour's arithmetic (arc lengths compared
    # modulo the track length, on the track)
    on = np.abs(e[1]) < 2.0
    L = np.float64(grids.track_length)
    d = np.abs(np.mod(a[0][on].astype(np.float64) - e[0][on] + L / 2, L) - L / 2)
    assert np.quantile(d, 0.999) < 1e-3
