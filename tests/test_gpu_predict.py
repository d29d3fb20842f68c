"""Prediction streaming on the device against the reference engine's own host re-simulation.

The reference's simulation engine (src/engine.cpp, unchanged, built in oracle/_ref against
the adapter's controllers.h, so its controllers are this library's) streams in every
MSG_STATE frame the trajectories its sendState (engine.cpp:55-264) re-simulates on the host
with its own model code, noise off: for MPPI the controller's plan under every hypothesis
from the state after the step, with branching; for PR-MPPI the new nominal under every
hypothesis and the robust plan under the last, from the state before the step. Replaying the
episode through the Python controllers (whose actions equal the engine's bit for bit, see
test_gpu_engine.py) and calling dr_mppi_predict / dr_prmppi_predict on the same inputs must
give the same branch records, stop reasons and times and ego actions, and positions within
FP32 rounding of the host's (the engine's host build evaluates the model without fused
multiply-adds, the device with them): 1e-4 relative or absolute.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

from conftest import O, drb
from test_gpu_engine import Rd, run_episode, to_state

pytestmark = pytest.mark.gpu
abi = drb.abi
S = drb.scenarios

TOL = 1e-4


def _frames_mppi(frames, n_agents):
    out = []
    for fr in frames:
        if struct.unpack_from("<i", fr)[0] != 1:
            continue
        r = Rd(fr)
        kind, step = r.i(), r.i()
        st = dict(step=step, pos=r.a(), vel=r.a(), S=r.a(), lat=r.a(), laps=r.a(), target=r.a(), action=r.a(), belief=r.a())
        st["fail"], st["eps"], st["eps_partial"], st["use_new"], st["cert"] = r.i(), r.f(), r.f(), r.i(), r.f()
        rows = []
        for _ in range(r.i()):
            init = r.a()
            bt, pt, pos, act = r.a(), r.a(), r.a(), r.a()
            rows.append(dict(init=int(init[0]), bt=int(bt[0]), pt=int(pt[0]), pos=pos.reshape(-1, 2 * n_agents), act=act.reshape(-1, 2),
                             reason=r.i(), time=r.i()))
        st["pred"] = rows
        out.append(st)
    return out


def _frames_pr(frames, n_agents):
    out = []
    for fr in frames:
        if struct.unpack_from("<i", fr)[0] != 1:
            continue
        r = Rd(fr)
        kind, step = r.i(), r.i()
        st = dict(step=step, pos=r.a(), vel=r.a(), S=r.a(), lat=r.a(), laps=r.a(), target=r.a(), action=r.a())
        st["prev_pos"], st["belief"], st["use_nom"], st["reset_nom"] = r.a(), r.a(), r.i(), r.i()
        rows = []
        for _ in range(r.i()):
            pos, act = r.a(), r.a()
            rows.append(dict(pos=pos.reshape(-1, 2 * n_agents), act=act.reshape(-1, 2), reason=r.i(), time=r.i()))
        st["pred"] = rows
        out.append(st)
    return out


def _close(a, b):
    return np.all(np.abs(a - b) <= TOL * np.maximum(1.0, np.abs(b)))


@pytest.mark.parametrize("gap", [None, 1.2])
def test_mppi_predictions_match_reference_engine(gpu, gap):
    """gap: start the ego that many metres of arc behind the opponent, close enough for the
    opponent's blocking to tell the hypotheses apart, so that the predictions branch."""
    sc = S.strat_race(use_splines=True, K=2048, T=40, n_verif=4096)
    if gap is not None:
        sc.state = S.initial_state(sc.grids, S._start_indices(sc.grids, 3.0, gap, 0), 1)
    frames = _frames_mppi(run_episode(sc, sc.mppi, 12), 2)
    assert len(frames) >= 3
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed)
    ctl.engine = object()
    worst = 0.0
    n_branch = 0
    for k, cur in enumerate(frames):
        if k > 0:
            prev = frames[k - 1]
            ctl.h_belief = prev["belief"].astype(np.float32)
            a = ctl.getControl(to_state(prev))
            assert np.array_equal(a, cur["action"]), f"step {k}: the replay left the engine's episode"
        pred = ctl.predict(to_state(cur), cur["belief"].astype(np.float32))
        for th, ref in enumerate(cur["pred"]):
            assert pred["init_branch"][th] == ref["init"], (k, th)
            assert pred["branching_time"][th] == ref["bt"] and pred["branch"][th] == ref["pt"], (k, th, pred["branch"][th], ref["pt"])
            assert pred["stop_reason"][th] == ref["reason"] and pred["stop_time"][th] == ref["time"], (k, th)
            assert np.array_equal(pred["actions"][th], ref["act"]), (k, th)
            assert _close(pred["positions"][th], ref["pos"]), (k, th, np.max(np.abs(pred["positions"][th] - ref["pos"])))
            worst = max(worst, float(np.max(np.abs(pred["positions"][th] - ref["pos"]))))
            n_branch += int(ref["pt"] != 0)
    print(f"{len(frames)} frames x {len(frames[0]['pred'])} hypotheses; largest position difference {worst:.2e}; rows that branched {n_branch}")


def test_mppi_prediction_branches_like_reference_host_model(gpu):
    """The engine's MPPI prediction loop (engine.cpp:96-166) restated here over the
    reference's own host model (environmentStep, oracle/_ref), on a plan that pushes the ego
    at an opponent 1.2 m ahead, so that the hypotheses separate and the predictions branch:
    dr_mppi_predict gives the same branch, branching time, stop reason and time and ego
    actions, and positions within FP32 rounding."""
    sc = S.strat_race(use_splines=False, K=512, T=40, n_verif=1024)
    sc.state = S.initial_state(sc.grids, S._start_indices(sc.grids, 3.0, 1.2, 0), 1)
    c = sc.mppi
    T, nth, nbp = c.n_timesteps, sc.n_theta, sc.n_theta + 1
    st0 = sc.state
    d = np.array([st0.pos[2] - st0.pos[0], st0.pos[3] - st0.pos[1]], np.float64)
    plan = np.broadcast_to(d / np.linalg.norm(d) * 4.0, (nbp, T, 2)).astype(np.float32).copy()
    ctl = drb.controllers.MPPIController(sc.env, c, sc.seed, nominal=plan)
    belief = sc.belief()
    pred = ctl.predict(sc.state, belief)
    ref = O.ref(O.ref_variant_name(nth, False))
    minc = float(np.float32(c.min_confidence))
    branched = 0
    for th in range(nth):
        st = drb.abi.dr_sim_state.from_buffer_copy(sc.state)
        bel = np.zeros(drb.abi.DR_MAX_THETA, np.float32)
        bel[:nth] = belief
        first = next((k + 1 for k in range(nth) if bel[k] > np.float32(minc)), 0)
        pt, bt, t_origin = first, (-1 if first == 0 else 0), 0
        stop_reason, stop_time = 3, -1
        pos = np.zeros((T, 4), np.float32)
        acts = np.zeros((T, 2), np.float32)
        for t in range(T):
            a = plan[pt, t - t_origin].copy()
            acts[t] = a
            term = ref.refh_env_step(C.byref(sc.env), th, O._f(a), C.byref(st), O._f(bel), 1, 0, minc, 0, 0, sc.seed, 0, t)
            npt = next((k + 1 for k in range(nth) if bel[k] > np.float32(minc)), 0)
            if pt == 0 and npt != 0:
                pt, bt, t_origin = npt, t + 1, t + 1
            pos[t] = np.array(st.pos[:4], np.float32)
            if term != 0:
                stop_reason, stop_time = {1: 0, 2: 1, 3: 2}[term], t
                pos[t + 1:] = pos[t]
                break
        branched += int(pt != 0)
        assert pred["branch"][th] == pt and pred["branching_time"][th] == bt, (th, pred["branch"][th], pt, pred["branching_time"][th], bt)
        assert pred["stop_reason"][th] == stop_reason and pred["stop_time"][th] == stop_time, th
        assert np.array_equal(pred["actions"][th], acts), th
        assert _close(pred["positions"][th], pos), (th, np.max(np.abs(pred["positions"][th] - pos)))
    assert branched > 0, "the case must branch"
    print(f"hypotheses that branched {branched} of {nth}; branching times {pred['branching_time']}")


def test_prmppi_predictions_match_reference_engine(gpu):
    sc = S.strat_race(use_pr=True, K=2048, T=40)
    frames = _frames_pr(run_episode(sc, sc.prmppi, 10), 2)
    assert len(frames) >= 3
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed)
    ctl.engine = object()
    worst = 0.0
    for k in range(1, len(frames)):
        prev, cur = frames[k - 1], frames[k]
        ctl.h_belief = prev["belief"].astype(np.float32)
        prev_state = to_state(prev)
        a = ctl.getControl(prev_state)
        assert np.array_equal(a, cur["action"]), f"step {k}: the replay left the engine's episode"
        pred = ctl.predict(prev_state)
        assert len(cur["pred"]) == sc.n_theta + 1
        for j, ref in enumerate(cur["pred"]):
            assert pred["stop_reason"][j] == ref["reason"] and pred["stop_time"][j] == ref["time"], (k, j)
            assert np.array_equal(pred["actions"][j], ref["act"]), (k, j)
            assert _close(pred["positions"][j], ref["pos"]), (k, j, np.max(np.abs(pred["positions"][j] - ref["pos"])))
            worst = max(worst, float(np.max(np.abs(pred["positions"][j] - ref["pos"]))))
    print(f"{len(frames) - 1} steps x {sc.n_theta + 1} rows; largest position difference {worst:.2e}")


def test_batch_predictions_on_device_equal_single(gpu):
    """dr_mppi_batch_predict_device after device-resident steps equals dr_mppi_predict of
    the same controllers stepped through the host."""
    import torch

    scs = [S.circle_race(agent=a, K=512, T=32 + 8 * a, n_verif=512) for a in range(3)]
    dev = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    host = [drb.controllers.MPPIController(s.env, s.mppi, s.seed) for s in scs]
    batch = drb.controllers.MPPIBatch(dev)
    n, nth, Tmax = len(scs), scs[0].n_theta, max(s.mppi.n_timesteps for s in scs)
    st_bytes = bytes((type(scs[0].state) * n)(*[s.state for s in scs]))
    st_dev = torch.frombuffer(bytearray(st_bytes), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    for i, s in enumerate(scs):
        bel[i, :nth] = s.belief()
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    for c in host:
        c.engine = object()
    for _ in range(2):
        batch.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        for c, s in zip(host, scs):
            c.getControl(s.state)
    pos = torch.zeros((n * nth, Tmax, 4), dtype=torch.float32, device="cuda")
    act = torch.zeros((n * nth, Tmax, 2), dtype=torch.float32, device="cuda")
    rec = torch.zeros((n * nth, abi.DR_PREDICT_RECORD), dtype=torch.int32, device="cuda")
    cost = torch.zeros(n * nth, dtype=torch.float32, device="cuda")
    abi.check(abi.lib().dr_mppi_batch_predict_device(batch._b, st_dev.data_ptr(), bel_dev.data_ptr(), pos.data_ptr(), act.data_ptr(), rec.data_ptr(),
                                                     cost.data_ptr(), Tmax), "batch_predict_device")
    torch.cuda.synchronize()
    pos, act, rec, cost = pos.cpu().numpy(), act.cpu().numpy(), rec.cpu().numpy(), cost.cpu().numpy()
    for i, (c, s) in enumerate(zip(host, scs)):
        p = c.predict(s.state, s.belief())
        T = s.mppi.n_timesteps
        rows = slice(i * nth, (i + 1) * nth)
        assert np.array_equal(pos[rows, :T], p["positions"])
        assert np.array_equal(act[rows, :T], p["actions"])
        assert np.array_equal(rec[rows, 3], p["stop_reason"]) and np.array_equal(rec[rows, 4], p["stop_time"])
        assert np.array_equal(cost[rows], p["cost"])
