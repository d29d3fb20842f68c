"""Drop-in check on the B200: the reference's own simulation engine (src/engine.cpp,
unchanged, built in oracle/_ref against the adapter's controllers.h) runs closed-loop
episodes on this library; replaying the states and beliefs it reports through the
Python controller classes (same C ABI, same seed) reproduces its actions bit for bit."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

from conftest import O, drb

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios


def _lib():
    path = O.REF_DIR / "libengine_dropin.so"
    if not path.exists():
        pytest.fail("oracle/_ref/libengine_dropin.so missing (make -C oracle engine)")
    L = C.CDLL(str(path))
    L.engine_run_episode.restype = C.c_int
    L.engine_run_episode.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t,
                                     C.POINTER(C.c_size_t), C.POINTER(C.c_int), C.c_int]
    return L


class Rd:
    def __init__(self, b):
        self.b, self.o = b, 0

    def i(self):
        v = struct.unpack_from("<i", self.b, self.o)[0]
        self.o += 4
        return v

    def f(self):
        v = struct.unpack_from("<f", self.b, self.o)[0]
        self.o += 4
        return v

    def a(self):
        n = self.i()
        v = np.frombuffer(self.b, "<f4", n, self.o).copy()
        self.o += 4 * n
        return v


def run_episode(sc, cont_cfg, steps):
    import drone_race_b200.protocol as P

    env_f = P.pack_env(sc.env, sc.grids, sc.seed, sc.true_theta)
    cont_f = P.pack_controller(cont_cfg)
    st_f = P.pack_state(sc.state, sc.env.n_opp)
    cap = 64 << 20
    out = (C.c_uint8 * cap)()
    n, nf = C.c_size_t(), C.c_int()
    rc = _lib().engine_run_episode(env_f, len(env_f), cont_f, len(cont_f), st_f, len(st_f), steps, out, cap, C.byref(n), C.byref(nf), 1)
    assert rc == 0
    return P.split_frames(bytes(out[: n.value]))


def parse_state(fr, n_theta, pr=False):
    r = Rd(fr)
    kind, step = r.i(), r.i()
    st = dict(kind=kind, step=step, pos=r.a(), vel=r.a(), S=r.a(), lat=r.a(), laps=r.a(), target=r.a(), action=r.a())
    if not pr:
        st["belief"] = r.a()
        st["fail"] = r.i()
        st["eps"] = r.f()
        st["eps_partial"] = r.f()
        st["use_new"] = r.i()
        st["cert"] = r.f()
    else:
        st["prev_pos"] = r.a()
        st["belief"] = r.a()
        st["use_nom"] = r.i()
        st["reset_nom"] = r.i()
    return st


def to_state(d) -> abi.dr_sim_state:
    s = abi.dr_sim_state()
    for i, v in enumerate(d["pos"]):
        s.pos[i] = float(v)
    for i, v in enumerate(d["vel"]):
        s.vel[i] = float(v)
    for a in range(len(d["S"])):
        s.S[a] = float(d["S"][a])
        s.lat_dist[a] = float(d["lat"][a])
        s.laps[a] = int(d["laps"][a])
    return s


def test_reference_engine_drives_mppi_dropin(gpu):
    sc = S.strat_race(use_splines=True, K=4096, T=40, n_verif=8192)
    steps = 25
    frames = run_episode(sc, sc.mppi, steps)
    states = [parse_state(f, 2) for f in frames if struct.unpack_from("<i", f)[0] == 1]
    assert len(states) >= 2 and struct.unpack_from("<i", frames[-1])[0] == 3  # MSG_DONE last
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed)
    ctl.engine = object()
    for k in range(1, len(states)):
        prev, cur = states[k - 1], states[k]
        ctl.h_belief = prev["belief"].astype(np.float32)
        a = ctl.getControl(to_state(prev))
        assert np.array_equal(a, cur["action"]), f"step {k}: {a} vs {cur['action']}"
        assert int(ctl.failCount.sum()) == cur["fail"]
        assert int(ctl.useNewPlan) == cur["use_new"]
        assert np.float32(ctl.epsilon) == np.float32(cur["eps"])


def test_reference_engine_drives_prmppi_dropin(gpu):
    sc = S.strat_race(use_pr=True, K=2048, T=40)
    steps = 15
    frames = run_episode(sc, sc.prmppi, steps)
    states = [parse_state(f, 2, pr=True) for f in frames if struct.unpack_from("<i", f)[0] == 1]
    assert len(states) >= 2 and struct.unpack_from("<i", frames[-1])[0] == 3
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed)
    ctl.engine = object()
    for k in range(1, len(states)):
        prev, cur = states[k - 1], states[k]
        ctl.h_belief = prev["belief"].astype(np.float32)
        a = ctl.getControl(to_state(prev))
        assert np.array_equal(a, cur["action"]), f"step {k}"
        assert int(ctl.useNomPlan) == cur["use_nom"] and int(ctl.resetNom) == cur["reset_nom"]
