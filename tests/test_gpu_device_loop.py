"""The device tail of the control step (finish_kernels.cu) and the device-resident closed
loop: Clopper-Pearson bounds on the device against the host's, device-resident control
steps against host steps of the same controllers, and a closed loop of control steps
and true-dynamics steps run entirely on the device against the same loop driven by the
host."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import drb
import helpers as H

pytestmark = pytest.mark.gpu

abi = drb.abi
S = drb.scenarios


def _torch():
    import torch

    return torch


def test_clopper_pearson_on_device_matches_host(gpu):
    rng = np.random.default_rng(0)
    for N in (1, 1024, 131072):
        k = np.unique(np.concatenate([np.arange(0, min(N, 40) + 1), rng.integers(0, N + 1, 200), [N - 1, N]])).astype(np.uint32)
        k = np.ascontiguousarray(k[k <= N])
        for alpha in (0.025, 0.05, 0.1):
            for upper in (0, 1):
                dev = np.zeros(k.size)
                host = np.zeros(k.size)
                abi.check(abi.lib().dr_debug_cp(abi.uptr(k), k.size, N, alpha, upper, dev.ctypes.data_as(C.POINTER(C.c_double))), "dr_debug_cp")
                abi.check(abi.lib().dr_debug_cp_host(abi.uptr(k), k.size, N, alpha, upper, host.ctypes.data_as(C.POINTER(C.c_double))),
                          "dr_debug_cp_host")
                # the two evaluate the same algorithm with the device's and the host's
                # lgamma / log1p / exp, whose last bits differ; an ill-conditioned quantile
                # (few failures out of 2^17) moves by up to ~1e-10 relative
                rel = np.abs(dev - host) / np.maximum(np.abs(host), 1e-300)
                assert rel.max() < 1e-9, (N, alpha, upper, rel.max(), k[rel.argmax()])


def _infos(buf, n):
    return (abi.dr_mppi_info * n).from_buffer_copy(buf.cpu().numpy().tobytes())


@pytest.mark.parametrize("use_splines", [True, False])
def test_device_steps_match_host_steps(gpu, use_splines):
    """Plans that fail verification part of the time (constant warm starts that crash), so that
    certification, plan choice, epsilon and the temperature adaptation all take both
    branches; the device tail must act exactly as the host tail."""
    torch = _torch()
    n = 3
    scs = [H.small_mppi(use_splines, K=512, T=40, n_verif=2048, seed=11 + a, noise=True) for a in range(n)]
    noms = []
    # with 2048 samples the certified loss is at least 0.0059 (the upper bound of no
    # failure at the first step): a threshold of 0.005 rejects every new plan, 0.01 accepts
    # all but those failing more than the previous; the constant warm starts crash, so the
    # histograms hold failures
    for sc, acc, eps in zip(scs, ([0.0, 0.0], [0.0, 3.0], [3.0, 0.0]), (0.005, 0.01, 0.01)):
        sc.mppi.max_verif_eps = eps
        noms.append(np.tile(np.array(acc, np.float32), (sc.n_theta + 1, sc.mppi.n_timesteps, 1)))
    A = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed, nominal=nm) for sc, nm in zip(scs, noms)]
    B = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed, nominal=nm) for sc, nm in zip(scs, noms)]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(B)
    states = [sc.state for sc in scs]
    beliefs = np.stack([sc.belief() for sc in scs])
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_sim_state * n)(*states))), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    bel[:, : beliefs.shape[1]] = beliefs
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    used = set()
    most = 0  # the largest failure count seen (1024 and above read the shared device table)
    for k in range(6):
        a_host = ba.step(states, beliefs)
        bb.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(a_host, act_dev.cpu().numpy()), k
        di = _infos(info_dev, n)
        for i in range(n):
            h, d = ba.infos[i], di[i]
            used.add(h.use_new_plan)
            most = max(most, int(h.fail_count_total))
            assert (h.use_new_plan, h.branch_idx, h.fail_count_total, h.nonfinite_costs) == (d.use_new_plan, d.branch_idx, d.fail_count_total,
                                                                                            d.nonfinite_costs)
            assert h.inv_temperature == d.inv_temperature and h.min_cost == d.min_cost and h.nu == d.nu
            assert abs(h.epsilon - d.epsilon) <= 1e-9 * abs(h.epsilon)
            assert abs(h.epsilon_partial - d.epsilon_partial) <= 1e-9 * max(abs(h.epsilon_partial), 1e-300)
            assert abs(h.certified_loss - d.certified_loss) <= 1e-9
    print("plans kept:", sorted(used), "largest failure count:", most)
    assert used == {0, 1}  # both outcomes of the certification were exercised
    # a host step after device steps continues from the state the device carried
    a1 = ba.step(states, beliefs)
    a2 = bb.step(states, beliefs)
    assert np.array_equal(a1, a2)
    for c1, c2 in zip(A, B):
        assert np.array_equal(c1.h_nominal, c2.h_nominal)
        assert c1.invTemperature == c2.invTemperature


@pytest.mark.parametrize("use_splines", [True, False])
def test_device_tail_large_failure_counts(gpu, use_splines):
    """The ego drone starts 8 m off the track, so every verification sample of both plans
    fails at its first step and the failure counts reach V = 2048: the device tail reads the
    Clopper-Pearson bounds of those counts from the shared table of large counts and must
    act exactly as the host tail."""
    torch = _torch()
    n = 2
    scs = [H.small_mppi(use_splines, K=256, T=40, n_verif=2048, seed=21 + a, noise=True) for a in range(n)]
    states = []
    for sc in scs:
        st = abi.dr_sim_state.from_buffer_copy(sc.state)
        st.pos[0] += 8.0
        st.pos[1] += 8.0
        states.append(st)
    A = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    B = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(B)
    beliefs = np.stack([sc.belief() for sc in scs])
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_sim_state * n)(*states))), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    bel[:, : beliefs.shape[1]] = beliefs
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    most = 0
    for k in range(3):
        a_host = ba.step(states, beliefs)
        bb.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(a_host, act_dev.cpu().numpy()), k
        di = _infos(info_dev, n)
        for i in range(n):
            h, d = ba.infos[i], di[i]
            most = max(most, int(h.fail_count_total))
            assert (h.use_new_plan, h.branch_idx, h.fail_count_total) == (d.use_new_plan, d.branch_idx, d.fail_count_total)
            assert abs(h.epsilon - d.epsilon) <= 1e-9 * abs(h.epsilon)
            assert abs(h.epsilon_partial - d.epsilon_partial) <= 1e-9 * max(abs(h.epsilon_partial), 1e-300)
            assert abs(h.certified_loss - d.certified_loss) <= 1e-9
    print("largest failure count:", most)
    assert most >= 1024


def test_device_closed_loop_matches_host_loop(gpu):
    """Control steps and true-dynamics steps alternated on the device (no host
    synchronisation inside the loop) against the loop the host drives with
    dr_mppi_batch_step and dr_env_step."""
    torch = _torch()
    n, steps, seed = 3, 20, 1234
    scs = [S.circle_race(agent=a, K=256, T=32, n_verif=512) for a in range(n)]
    A = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    B = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(B)
    # host loop
    states = [abi.dr_sim_state.from_buffer_copy(sc.state) for sc in scs]
    bels = [np.zeros(abi.DR_MAX_THETA, np.float32) for _ in scs]
    for b, sc in zip(bels, scs):
        b[: sc.n_theta] = sc.belief()
    terms_h = []
    for t in range(steps):
        act = ba.step(states, np.stack([b[: scs[0].n_theta] for b in bels]))
        terms_h.append([drb.controllers.env_step(sc.env, 0, act[i], states[i], bels[i], True, seed, t + 1) for i, sc in enumerate(scs)])
    # device loop
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_sim_state * n)(*[sc.state for sc in scs]))), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    for i, sc in enumerate(scs):
        bel[i, : sc.n_theta] = sc.belief()
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    theta_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    term_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    terms_d = []
    for t in range(steps):
        bb.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        bb.env_step_device(theta_dev.data_ptr(), act_dev.data_ptr(), st_dev.data_ptr(), bel_dev.data_ptr(), True, seed, term_dev.data_ptr())
        torch.cuda.synchronize()  # the batch runs on its own stream
        terms_d.append(term_dev.cpu().numpy().tolist())
    torch.cuda.synchronize()
    assert terms_h == terms_d
    final = (abi.dr_sim_state * n).from_buffer_copy(st_dev.cpu().numpy().tobytes())
    for i in range(n):
        assert bytes(final[i]) == bytes(states[i]), i
        assert np.array_equal(bel_dev.cpu().numpy()[i], bels[i])


def test_gate_race_device_steps_match_host_steps(gpu):
    """The device tail on gate-race controllers (dr_gate_state records)."""
    torch = _torch()
    n = 2
    scs = [H.small_gate(False, K=512, T=40, n_verif=1024, seed=5 + a, noise=True) for a in range(n)]
    A = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    B = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(B)
    states = [sc.state for sc in scs]
    beliefs = np.stack([np.array(sc.env.init_belief[: sc.env.n_theta], np.float32) for sc in scs])
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_gate_state * n)(*states))), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    bel[:, : beliefs.shape[1]] = beliefs
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    for k in range(4):
        a_host = ba.step(states, beliefs)
        bb.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(a_host, act_dev.cpu().numpy()), k
        di = _infos(info_dev, n)
        for i in range(n):
            h, d = ba.infos[i], di[i]
            assert (h.use_new_plan, h.branch_idx, h.fail_count_total) == (d.use_new_plan, d.branch_idx, d.fail_count_total)
            assert h.inv_temperature == d.inv_temperature and h.nu == d.nu
            assert abs(h.epsilon - d.epsilon) <= 1e-9 * abs(h.epsilon)


def test_gate_race_device_closed_loop_matches_host_loop(gpu):
    """The gate race's closed loop on the device (gate_batch_env_step) against the loop
    driven by the host with dr_gate_mppi_batch_step and dr_gate_env_step."""
    torch = _torch()
    n, steps, seed = 2, 12, 77
    scs = [H.small_gate(False, K=256, T=32, n_verif=512, seed=5 + a, noise=True) for a in range(n)]
    A = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    B = [drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed) for sc in scs]
    ba, bb = drb.controllers.MPPIBatch(A), drb.controllers.MPPIBatch(B)
    nth = scs[0].env.n_theta
    states = [abi.dr_gate_state.from_buffer_copy(sc.state) for sc in scs]
    bels = [np.array(sc.env.init_belief[:nth], np.float32) for sc in scs]
    terms_h = []
    for t in range(steps):
        act = ba.step(states, np.stack(bels))
        row = []
        for i, sc in enumerate(scs):
            term, states[i], bels[i] = drb.controllers.gate_env_step(sc.env, 0, act[i], states[i], bels[i], True, seed, t + 1)
            row.append(term)
        terms_h.append(row)
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_gate_state * n)(*[sc.state for sc in scs]))), dtype=torch.uint8).cuda()
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    for i, sc in enumerate(scs):
        bel[i, :nth] = sc.env.init_belief[:nth]
    bel_dev = torch.from_numpy(bel).cuda()
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    theta_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    term_dev = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    terms_d = []
    for t in range(steps):
        bb.step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())
        bb.env_step_device(theta_dev.data_ptr(), act_dev.data_ptr(), st_dev.data_ptr(), bel_dev.data_ptr(), True, seed, term_dev.data_ptr())
        torch.cuda.synchronize()
        terms_d.append(term_dev.cpu().numpy().tolist())
    assert terms_h == terms_d
    final = (abi.dr_gate_state * n).from_buffer_copy(st_dev.cpu().numpy().tobytes())
    for i in range(n):
        assert bytes(final[i]) == bytes(states[i]), i
        assert np.array_equal(bel_dev.cpu().numpy()[i, :nth], bels[i])
