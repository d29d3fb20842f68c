#!/usr/bin/env python
"""Throughput of the MPPI control step on B200.

Workload (per GPU): 4 agents, each an MPPI controller with K = 4096 samples, horizon
H = 64 (dense controls), 2 opponent hypotheses, one policy opponent, plan verification
with V = 2^17 samples over 40 steps (the reference front-end's setting), on a seeded
synthetic track (closed Catmull-Rom through 12 control points jittered +-5 m around a
40 m circle). One control step = every agent's getControl once.

value : control steps/s with inputs resident in HBM (dr_mppi_batch_step_device: the
        whole control step on the device, its host tail included; CUDA events)
e2e   : control steps/s through the C ABI with host buffers (dr_mppi_batch_step: inputs
        copied from pinned host memory, results copied back, host tail included)

Multi-GPU: one process per GPU, each running its own 4-agent race (replicas, weak
scaling, no data-path collective); timing is the max over ranks.

--impl reference times the reference's own CPU implementation of the path (its model
functions compiled from the reference sources, oracle/_ref, OpenMP over all host
threads) on a bounded sample of the same workload. When a GPU is present it also
reports, as an extra field, the reference's own CUDA path (its kernels and its
MPPIController::getControl compiled from the reference sources) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "drone-race_b200"

AGENTS = 4
K = 4096
H = 64
N_THETA = 2
V = 2**17
VERIF_H = 40

# Algorithmic FP32 work of one environment step (unit = one (agent, sample, hypothesis,
# timestep) step), counted by running the oracle's model with an operation-counting
# scalar over 256 samples of this workload (oracle/port/opcount.cpp): every add, sub,
# mul, div, sqrt, exp, log, pow, min/max/abs/floor/copysign = 1 FLOP, comparisons not
# counted, and an operation repeated on the same operands within one step counted once
# (the reference evaluates 1323 ops per step as written; 652 / 571 are distinct).
# The verification shares the ego's moves across its samples (the ego draws no noise in
# this workload, so samples that took the same branch at the same step move it alike;
# mppi_ego_table computes them once per plan): counting each distinct operation once per
# step index over the samples (opcount dedup mode 2) leaves 337 FLOPs per sample-step.
# Work whose result nothing reads (a committed sample's belief update and the other
# hypotheses' actions, which the kernels skip) is left out too, and the track projection
# is counted as the kernels run it: the certified local search of its window, three to a
# few distances where the reference's scan takes 21 (the same sample; this workload's
# track certifies everywhere on it). That leaves 442.0 FLOPs per rollout step and 233.7
# per verification step (652.4 / 337.0 with the window scanned as the reference does).
# `python oracle/count_flops.py` reproduces every count of this file.
FLOPS_PER_ROLLOUT_STEP = 442.0    # MPPI rollout step (belief update over 2 hypotheses)
FLOPS_PER_VERIFY_STEP = 233.7     # verification step, ego moves shared across samples

# --workload gates: the same control step on the gate race (the reference's EnvDroneRace:
# one PID opponent with 2 hypotheses, 8 gates on a 30 x 20 m ellipse, 2 racelines), FLOPs
# per step counted the same way on oracle/port/gate_model.hpp (orc_gate_count_ops), the
# raceline walks without the margin scans the kernels skip where certified: 189.7 per
# rollout step, 117.8 per verification step (405.7 / 328.4 with the margins scanned as
# the reference does).
N_GATES = 8
GATE_FLOPS_PER_ROLLOUT_STEP = 189.7
GATE_FLOPS_PER_VERIFY_STEP = 117.8

# --workload grad: gradient-refined MPPI on the strategic race, a quarter of the samples
# (K = 1024) and one projected gradient step (--grad-steps) of the noise-free rollout objective after each
# update (dr_mppi_set_grad_refine), beside plain MPPI at K = 4096 in closed loop.
K_GRAD = 1024
GRAD_STEPS = 1
GRAD_STEP_SIZE = 0.05
# --workload pr: PR-MPPI (the reference's PRMPPIController) on the strategic race with the
# benchmark's PR configuration per agent: 8 opponent hypotheses (lateral aggressiveness
# U(0, 2) m, speed scale U(0.8, 1.2), belief ~ Dirichlet(1)), P = 8 sampled hypotheses,
# K = 2048, H = 64. FLOPs per PR rollout step (one hypothesis' policy, no belief update,
# PRMPPIstateCost and PRMPPIsafetyCost) counted like the others (orc_pr_count_ops), the
# projection as the kernels search it: 411.7 (623.5 with the window scanned as written).
K_PR, P_PR, NTH_PR = 2048, 8, 8
PR_FLOPS_PER_ROLLOUT_STEP = 411.7
# --workload races: many independent races of uneven sizes in one batch per control mode
# (scenarios.uneven_races: 256 races, U{1..8} agents each, K log-uniform [256, 16384],
# H in {32, 48, 64, 96}, tracks through U{6..16} points, dense and spline controls by
# race), verification of 4096 samples over min(40, H) steps per agent; one control step =
# every agent of every race advanced once. Measured with one CTA per tile, with persistent
# launches fed by the device work queue, and with the shapes the autotuner picks.
N_RACES = 256
V_RACES = 4096
WL = {"kind": "strat"}  # the workload of this run (set from --workload)


def _K() -> int:
    return K_GRAD if WL["kind"] == "grad" else K


def _flops():
    if WL["kind"] == "gates":
        return GATE_FLOPS_PER_ROLLOUT_STEP, GATE_FLOPS_PER_VERIFY_STEP
    return FLOPS_PER_ROLLOUT_STEP, FLOPS_PER_VERIFY_STEP


def _workload_name() -> str:
    if WL["kind"] == "pr":
        return f"prmppi_4x{P_PR}x{K_PR}x64_{NTH_PR}hyp"
    if WL["kind"] == "gates":
        return "gate_mppi_4x4096x64_8gates"
    if WL["kind"] == "grad":
        return f"grad_mppi_4x{K_GRAD}x64_{GRAD_STEPS}steps"
    return "mppi_4x4096x64"


def _unit() -> str:
    if WL["kind"] == "pr":
        return f"control steps/s (4 agents x PR-MPPI with P={P_PR} hypotheses x K={K_PR} x H=64, nominal and robust plans; all agents advanced once)"
    if WL["kind"] == "grad":
        return (f"control steps/s (4 agents x K={K_GRAD} x H=64 MPPI + {GRAD_STEPS} projected gradient steps, verification V=2^17 x 40, "
                "all agents advanced once; strategic race)")
    race = f"gate race, {N_GATES} gates" if WL["kind"] == "gates" else "strategic race"
    return f"control steps/s (4 agents x K=4096 x H=64 MPPI, verification V=2^17 x 40, all agents advanced once; {race})"


def _ref_variant(O) -> str:
    return "gate8_dense" if WL["kind"] == "gates" else O.ref_variant_name(N_THETA, False)

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu capture
# of each kernel on this workload (--quick --no-overlap, 3 steps); grids, plans and tile
# tables stay in L2, so DRAM traffic is spilled registers and first-touch reads, about 0.9
# MB per verification launch (both plans, with the ego tables).
TRAFFIC_PER_LAUNCH: dict[str, float] = {"verify": 855040.0, "rollout": 168960.0}


def _package():
    if "drone_race_b200" in sys.modules:
        return sys.modules["drone_race_b200"]
    spec = importlib.util.spec_from_file_location("drone_race_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["drone_race_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(rank: int):
    drb = _package()
    S = drb.scenarios
    if WL["kind"] == "gates":
        return [S.gate_race(agent=a, seed=rank, K=K, T=H, use_splines=False, n_verif=V, n_gates=N_GATES) for a in range(AGENTS)]
    return [S.circle_race(agent=a, seed=rank, K=_K(), T=H, use_splines=False, n_theta=N_THETA, n_verif=V) for a in range(AGENTS)]


class Clocks:
    """SM clocks and clock-event reasons sampled during the timed region: NVML read by a
    thread every few milliseconds, with one sample taken when the region starts and one when
    it ends, so that even a short region has samples (nvidia-smi polling as the fallback)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"), ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"), ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nv = None
        self.path = Path(f"/tmp/dr_clocks_{os.getpid()}.csv")
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = self._handle(pynvml, index)
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.bits = {name: getattr(pynvml, attr) for name, attr in self.REASONS}
        except Exception:
            self.nv = None

    @staticmethod
    def _handle(pynvml, index: int):
        """The NVML device of CUDA device `index` (matched by PCI bus id when torch has it)."""
        try:
            import torch

            bus = getattr(torch.cuda.get_device_properties(index), "pci_bus_id", None)
            dom = getattr(torch.cuda.get_device_properties(index), "pci_domain_id", 0)
            dev = getattr(torch.cuda.get_device_properties(index), "pci_device_id", None)
            if bus is not None and dev is not None:
                return pynvml.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dev:02x}.0")
        except Exception:
            pass
        return pynvml.nvmlDeviceGetHandleByIndex(index)

    def _sample(self):
        nv = self.nv
        sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
        r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
        self.samples.append((sm, {name for name, bit in self.bits.items() if r & bit}))

    def _loop(self):
        while not self.done.wait(0.005):
            try:
                self._sample()
            except Exception:
                return

    def start(self):
        if self.nv is not None:
            import threading

            self.samples = []
            self.done = threading.Event()
            try:
                self._sample()
            except Exception:
                self.nv = None
            else:
                self.thread = threading.Thread(target=self._loop, daemon=True)
                self.thread.start()
                return
        q = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.nv is not None:
            self.done.set()
            self.thread.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
            sm = [x for x, _ in self.samples]
            reasons = set().union(*(r for _, r in self.samples)) if self.samples else set()
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.mx, "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        try:
            self.path.unlink()
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def _dist():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def _max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """Max of a per-rank time over all ranks (the multi-GPU timing rule)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_baseline_reference(scs, target_s: float = 10.0, max_reps: int = 100000, k_s: int = 4096, v_s: int = 32768, fp64: bool = True) -> dict:
    """The reference's CPU path (its model functions from oracle/_ref, OpenMP) on a bounded
    sample of one agent's control step, scaled to the 4-agent control step. The sample
    controls agent 0 from its start state with an all-zero plan (the plan only steers the
    ego drone; none of its verification samples fails within the 40 steps, so the sample
    does the full horizon of work)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O

    drb = _package()
    O.set_abi(drb.abi)
    variant = _ref_variant(O)
    kind = "reference"
    if not O.ref_available(variant):
        kind = "port"
    threads = os.cpu_count() or 1
    sc = scs[0]
    c = sc.mppi
    belief = sc.belief()
    # sample: k_s rollout samples and v_s verification samples
    c_small = type(c).from_buffer_copy(c)
    c_small.n_samples = k_s
    c_small.n_verif_samples = v_s
    sc.mppi = c_small
    nominal = np.zeros((N_THETA + 1, H, 2), np.float32)
    noise = O.mppi_noise(sc, 0)
    t0 = time.perf_counter()
    reps = 0
    t_roll = t_ver = 0.0
    while True:
        a = time.perf_counter()
        if kind == "reference":
            O.mppi_rollout(sc, belief, nominal, noise, None, 0, impl=variant, nthreads=threads)
        else:
            O.mppi_rollout(sc, belief, nominal, noise, None, 0, prec=32)
        b = time.perf_counter()
        if kind == "reference":
            O.mppi_verify(sc, belief, nominal, 0, 0, impl=variant, nthreads=threads)
        else:
            O.mppi_verify(sc, belief, nominal.astype(np.float64), 0, 0, prec=32)
        e = time.perf_counter()
        t_roll += b - a
        t_ver += e - b
        reps += 1
        if e - t0 > target_s or reps >= max_reps:
            break
    t_roll /= reps
    t_ver /= reps
    # scale: rollout work ~ samples, verification ~ samples (x2 plans); 4 agents
    step_s = AGENTS * (t_roll * (_K() / k_s) + 2 * t_ver * (V / v_s))
    sample = (f"1 agent: rollout of {k_s} samples x {N_THETA} hypotheses x {H} steps and one verification pass of {v_s} samples x {VERIF_H} steps, "
              f"{reps} repetitions ({time.perf_counter() - t0:.1f} s), scaled to 4 agents x K={_K()} and 2 x V={V}")
    if not fp64:
        sc.mppi = c
        return {"value": 1.0 / step_s, "unit": "control_steps/s", "cores": threads, "kind": kind, "sample": sample, "ms_per_control_step": step_s * 1e3}
    # the FP64 transcription of the same model (the oracle port at double precision,
    # OpenMP over all host threads) on a quarter of the sample, a few seconds
    f0 = time.perf_counter()
    f_reps = 0
    f_roll = f_ver = 0.0
    c_q = type(c).from_buffer_copy(c_small)
    c_q.n_samples = k_s // 4
    c_q.n_verif_samples = v_s // 4
    sc.mppi = c_q
    noise_q = O.mppi_noise(sc, 0)
    while True:
        a = time.perf_counter()
        O.mppi_rollout(sc, belief, nominal, noise_q, None, 0, prec=64)
        b = time.perf_counter()
        O.mppi_verify(sc, belief, nominal.astype(np.float64), 0, 0, prec=64)
        e = time.perf_counter()
        f_roll += b - a
        f_ver += e - b
        f_reps += 1
        if e - f0 > target_s / 3 or f_reps >= max_reps:
            break
    sc.mppi = c
    f_step = AGENTS * (f_roll / f_reps * (_K() / (k_s // 4)) + 2 * f_ver / f_reps * (V / (v_s // 4)))
    fp64 = {"value": 1.0 / f_step, "unit": "control_steps/s", "cores": threads, "kind": "port (FP64 transcription)",
            "sample": f"1 agent: rollout of {k_s // 4} samples and one verification pass of {v_s // 4} samples, {f_reps} repetitions, scaled likewise"}
    return {"value": 1.0 / step_s, "unit": "control_steps/s", "cores": threads, "kind": kind, "sample": sample,
            "ms_per_control_step": step_s * 1e3, "fp64_transcription": fp64}


def _race_cost_step(sc, st) -> float:
    """stateCost (costs.cuh:7-28) of a true state of the strategic race, undiscounted."""
    e, c = sc.env, sc.mppi
    r = e.drone_radius
    n = e.n_opp + 1
    p = np.array(st.pos[: 2 * n], np.float64).reshape(n, 2)
    opp_won = any(st.laps[o] >= e.n_win_laps for o in range(1, n))
    bd = min(min(np.linalg.norm(p[o] - p[0]) for o in range(1, n)) - r, e.track_width - abs(st.lat_dist[0]))
    winner = st.laps[0] >= e.n_win_laps or any(abs(st.lat_dist[o]) > e.track_width - r for o in range(1, n))
    cost = 0.0
    if bd < c.boundary_threshold_factor * r:
        cost += c.boundary_cost * (bd / r) ** 2
    if bd < r * c.coll_dist_factor:
        cost += c.outside_cost
    if opp_won:
        cost += c.opp_win_cost
    if winner:
        cost -= c.win_cost
    return cost


def closed_loop_compare(n_steps: int = 500) -> dict:
    """Gradient-refined MPPI (K = K_GRAD, GRAD_STEPS steps) against plain MPPI (K = 4096)
    in closed loop: each of the 4 benchmark agents races its opponent for n_steps control
    steps (true dynamics on the device, true hypothesis 0, belief updated), the race cost
    of the executed trajectory (sum of stateCost plus finalCost) and the wall time per
    control step (host loop: getControl + environment step) recorded for either arm."""
    drb = _package()
    import drone_race_b200.controllers as ctl_mod

    abi = drb.abi
    arms = {}
    for name, k, g in (("plain", K, 0), ("grad", K_GRAD, GRAD_STEPS)):
        costs, progress, ms, outcome, improved = [], [], [], [], 0
        for a in range(AGENTS):
            sc = drb.scenarios.circle_race(agent=a, seed=0, K=k, T=H, use_splines=False, n_theta=N_THETA, n_verif=V)
            ctl = ctl_mod.MPPIController(sc.env, sc.mppi, sc.seed)
            ctl.engine = object()
            if g:
                ctl.set_grad_refine(g, GRAD_STEP_SIZE, 0)
            st = abi.dr_sim_state.from_buffer_copy(sc.state)
            bel = np.zeros(abi.DR_MAX_THETA, np.float32)
            bel[: N_THETA] = sc.belief()
            run_cost, term, t = 0.0, 0, 0
            t0 = time.perf_counter()
            for t in range(n_steps):
                ctl.h_belief[:] = bel[: N_THETA]
                act = ctl.getControl(st)
                improved += int(g > 0 and ctl.info.grad_best_step > 0)
                term = ctl_mod.env_step(sc.env, 0, act, st, bel, True, sc.seed, t)
                run_cost += _race_cost_step(sc, st)
                if term:
                    break
            ms.append((time.perf_counter() - t0) / (t + 1) * 1e3)
            prog = st.S[0] / sc.env.track_length + st.laps[0]
            costs.append(run_cost - sc.mppi.final_adv_weight * prog)
            progress.append(prog)
            outcome.append({0: "running", 1: "lost", 2: "won", 3: "opponent won"}.get(term, str(term)) + f" after {t + 1} steps")
            ctl.close()
        arms[name] = {"K": k, "grad_steps": g, "race_cost_mean": float(np.mean(costs)), "race_costs": costs, "progress_mean": float(np.mean(progress)),
                      "ms_per_control_step_wall": float(np.mean(ms)), "outcomes": outcome}
        if g:
            arms[name]["steps_refined"] = improved
    arms["what"] = (f"{AGENTS} agents x up to {n_steps} closed-loop control steps each; race cost = sum of stateCost over the executed states + "
                    "finalCost of the last (lower is better); the episode ends at a terminal state")
    return arms


def run_ours(args) -> None:
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    drb = _package()
    import drone_race_b200.controllers as ctl_mod

    abi = drb.abi
    scs = workload(rank)

    def make_set(shapes=None):
        """A fresh batch of the workload's controllers (same scenarios and seeds). The
        device-resident timing, the end-to-end timing and the per-kernel passes each run on
        their own set, after the same number of warm-up steps, so that they all start from
        the same controller state (the per-step work drifts as the plans evolve)."""
        stream = torch.cuda.Stream()  # non-default stream: the batch captures a CUDA graph on it
        ctls = [ctl_mod.MPPIController(s.env, s.mppi, s.seed, device=local, stream=stream.cuda_stream) for s in scs]
        if WL["kind"] == "grad":
            for c in ctls:
                c.set_grad_refine(GRAD_STEPS, GRAD_STEP_SIZE, shapes["grad_ckpt"] if shapes else 0)
        batch = ctl_mod.MPPIBatch(ctls, stream=stream.cuda_stream)
        if args.no_overlap:
            batch.set_overlap(False)
        if args.side_verify is not None:
            batch.set_side_verify(args.side_verify)
        if args.pdl:
            batch.set_pdl(True)
        if shapes:
            batch.set_persistent(shapes["rollout_ctas_per_sm"], shapes["verify_ctas_per_sm"], bool(shapes["rollout_lockstep"]))
        return stream, ctls, batch

    stream, ctls, batch = make_set()
    n = len(ctls)
    states = [s.state for s in scs]
    beliefs = np.stack([s.belief() for s in scs])
    # device-resident inputs
    st_bytes = bytes((type(states[0]) * n)(*states))
    st_dev = torch.frombuffer(bytearray(st_bytes), dtype=torch.uint8).to("cuda")
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    bel[:, :N_THETA] = beliefs
    bel_dev = torch.from_numpy(bel).to("cuda")
    act_dev = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    info_dev = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def dev_step(b=None):
        # the whole control step on the device, its tail included (dr_mppi_batch_step_device)
        (b or batch).step_device(st_dev.data_ptr(), bel_dev.data_ptr(), act_dev.data_ptr(), info_dev.data_ptr())

    # ---- device-resident throughput -------------------------------------------------------
    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize()
    # launch shapes (grid, lockstep, checkpoint stride) chosen by the library's autotuner on
    # this batch, before the timed region
    tune = batch.autotune(10)
    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dev_step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    _barrier(world)
    ms = e0.elapsed_time(e1)
    ms = _max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)

    # ---- end to end through the C ABI with host buffers -----------------------------------
    # a second set of controllers, warmed up by as many steps as the first before its timed
    # region and launched with the shapes the autotuner chose
    e2e_s = None
    h2d = d2h = 0
    if not args.quick:
        _, ctls_h, batch_h = make_set(tune)
        for c in ctls_h:
            c.engine = object()
        for _ in range(2 * args.warmup):
            batch_h.step(states, beliefs)
        torch.cuda.synchronize()
        _barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            batch_h.step(states, beliefs)
        t1 = time.perf_counter()
        _barrier(world)
        e2e_s = _max_over_ranks(max(t1 - t0, 1e-9), world)
        for c in ctls_h:
            a, b = C.c_size_t(), C.c_size_t()
            abi.lib().dr_mppi_io_bytes(c.handle, C.byref(a), C.byref(b))
            h2d += a.value
            d2h += b.value
        batch_h.close()
        for c in ctls_h:
            c.close()

    # ---- per-kernel times, the streams' schedule and the roofline --------------------------
    # A third set, warmed up like the first, with CUDA events between the kernels (launched
    # directly, not replayed from the graph). First a pass with the verification of both
    # plans in one launch on the main stream (the kernels one at a time: in the overlapped
    # schedule the two verification launches share the SMs with each other and with the
    # rollout, so their event durations are not per-kernel times), then the default
    # overlapped schedule.
    _, ctls_p, batch_p = make_set(tune)
    for _ in range(2 * args.warmup):
        dev_step(batch_p)
    torch.cuda.synchronize()
    serial_steps = max(10, min(50, args.steps))
    kt_serial = None
    if not args.no_overlap:
        batch_p.set_overlap(False)
        batch_p.set_profiling(True)
        for _ in range(serial_steps):
            dev_step(batch_p)
        torch.cuda.synchronize()
        kt_serial = batch_p.kernel_times()
        batch_p.set_profiling(False)
        batch_p.set_overlap(True)
    batch_p.set_profiling(True)
    for _ in range(args.steps):
        dev_step(batch_p)
    torch.cuda.synchronize()
    kt = batch_p.kernel_times()
    timeline = {k: [round(a, 4), round(b, 4)] for k, (a, b) in batch_p.kernel_timeline().items()}
    batch_p.set_profiling(False)
    if kt_serial is None:
        kt_serial, serial_steps = kt, args.steps
    units = {"rollout": AGENTS * _K() * N_THETA * H, "verify": AGENTS * 2 * V * VERIF_H}
    flops_unit = dict(zip(("rollout", "verify"), _flops()))
    dom = max(kt_serial, key=kt_serial.get) if kt_serial else None
    roof = roof_step = None
    if dom in units and clk.get("sm_mhz"):
        peak = 2 * 128 * 148 * clk["sm_mhz"] * 1e6 / 1e12
        achieved = units[dom] * flops_unit[dom] / (kt_serial[dom] / 1e3) / 1e12
        roof = {"bound": "fp32", "kernel": f"mppi_verify ({dom})" if dom == "verify" else f"mppi_{dom}", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": TRAFFIC_PER_LAUNCH.get(dom) if WL["kind"] == "strat" else None,
                "peak_source": "FP32 FMA rate of 148 SMs x 128 lanes at the median SM clock sampled during the timed region (MEASURED_PEAKS.json has no FP32 figure)",
                "units_per_launch": units[dom], "flops_per_unit": flops_unit[dom], "kernel_ms": kt_serial[dom],
                "measured": f"CUDA events around each launch on its stream, {serial_steps} steps with both plans verified in one launch"}
        step_flops = sum(units[k] * flops_unit[k] for k in units)
        ach_step = step_flops / (ms_per_step / 1e3) / 1e12
        roof_step = {"bound": "fp32", "achieved": ach_step, "peak": peak, "unit": "TFLOP/s", "frac": ach_step / peak,
                     "scope": "all FP32 work of one control step (rollout + both verifications) / device step time of the timed region"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.quick:
        cpu = cpu_baseline_reference(scs)
        cpu.pop("ms_per_control_step", None)

    rollout_steps = AGENTS * _K() * N_THETA * H
    line = {
        "metric": "control_steps_per_s",
        "value": value,
        "unit": _unit(),
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded tracks and states; no dataset)",
        "config": {"workload": _workload_name(), "agents": AGENTS, "K": _K(), "H": H, "n_theta": N_THETA, "n_opp": 1, "controls": "dense",
                   "verif_samples": V, "verif_horizon": VERIF_H, "parallelism": f"replicas x{world}",
                   "l2": "working set per step < L2; steps are dependent control steps of the same controllers"},
        "rollout_steps_per_s": world * rollout_steps * args.steps / (ms / 1e3),
        "verify_steps_per_s": world * AGENTS * 2 * V * VERIF_H * args.steps / (ms / 1e3),
        "kernel_ms": kt,
        "kernel_timeline_ms": timeline,
        "kernel_ms_serial": kt_serial,
        "e2e": None if e2e_s is None else {"value": world * args.steps / e2e_s, "unit": "control steps/s", "h2d_bytes_per_step": h2d,
                                           "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s / args.steps * 1e3},
        "gpu_launches": len(kt) * args.steps,
        "autotune": {"rollout_ctas_per_sm": tune["rollout_ctas_per_sm"], "rollout_lockstep": tune["rollout_lockstep"],
                     "verify_ctas_per_sm": tune["verify_ctas_per_sm"], "grad_ckpt": tune["grad_ckpt"],
                     "rollout_ms": {f"{c}x{l}": v for (c, l), v in tune["rollout"].items()}, "verify_ms": tune["verify"], "grad_ms": tune["grad"]},
        "roofline": roof,
        "roofline_step": roof_step,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if WL["kind"] == "grad" and rank == 0 and world == 1 and not args.quick:
        line["grad_vs_plain"] = closed_loop_compare()
    if rank == 0:
        print(json.dumps(line), flush=True)
    for b_, cs_ in ((batch, ctls), (batch_p, ctls_p)):
        b_.close()
        for c in cs_:
            c.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def reference_cuda_timing(scs, warmup: int = 3, steps: int = 20) -> dict | None:
    """The reference's own CUDA path on this GPU (oracle/_ref, compiled from the reference
    sources for sm_100a, N_OPP 1, N_TRUE_MODELS 2, dense controls), 4 controllers on the
    benchmark track: (i) its kernel sequence of one MPPI update per agent (noise, rollout,
    aggregation, masked min, weighted average, clamp; CUDA events), (ii) its full
    MPPIController::getControl per agent, verification of both plans included (wall time
    with the device synchronised). None without a GPU or without the compiled reference."""
    try:
        import torch

        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O

    drb = _package()
    O.set_abi(drb.abi)
    variant = _ref_variant(O)
    if not O.ref_available(variant):
        return None
    sc = scs[0]
    out = (C.c_double * 2)()
    rc = O.ref(variant).refc_mppi_time(C.byref(sc.env), C.byref(sc.mppi), C.byref(sc.state), AGENTS, warmup, steps, out)
    if rc != 0:
        return {"error": f"reference CUDA timing failed with status {rc}"}
    return {"kernels_ms_per_step": out[0], "getcontrol_ms_per_step": out[1], "control_steps_per_s": 1e3 / out[1],
            "kernels_only_steps_per_s": 1e3 / out[0], "steps": steps, "warmup": warmup,
            "what": "reference CUDA kernels built from its sources: (i) noise+rollout+aggregate+min+weighted average+clamp per agent, "
                    "CUDA events; (ii) MPPIController::getControl per agent incl. verification, wall clock"}


def _pr_workload(rank: int):
    drb = _package()
    return [drb.scenarios.robust_race(agent=a, seed=rank, K=K_PR, T=H, P=P_PR, n_theta=NTH_PR) for a in range(AGENTS)]


def cpu_baseline_pr(scs, target_s: float = 10.0, max_reps: int = 100000, k_s: int = 512) -> dict:
    """The reference's CPU PR-MPPI rollout (its model functions, oracle/_ref, OpenMP) on a
    bounded sample of one agent: k_s samples x P hypotheses x nominal and robust plans x
    H steps, scaled to the 4-agent step (the rollout is the PR step's work)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O

    drb = _package()
    O.set_abi(drb.abi)
    variant = O.ref_variant_name(NTH_PR, True)
    kind = "reference" if O.ref_available(variant) else "port"
    threads = os.cpu_count() or 1
    sc = scs[0]
    c = sc.prmppi
    c_small = type(c).from_buffer_copy(c)
    c_small.n_samples = k_s
    sc.prmppi = c_small
    noise = O.pr_noise(sc, 0)
    thetas = O.pr_thetas(sc, 0, sc.belief())
    nom = np.zeros((H, 2), np.float32)
    t0 = time.perf_counter()
    reps = 0
    while True:
        if kind == "reference":
            O.pr_rollout(sc, nom, nom, noise, thetas, 0, impl=variant, nthreads=threads)
        else:
            O.pr_rollout(sc, nom.astype(np.float64), nom.astype(np.float64), noise, thetas, 0, prec=32)
        reps += 1
        if time.perf_counter() - t0 > target_s or reps >= max_reps:
            break
    el = (time.perf_counter() - t0) / reps
    sc.prmppi = c
    step_s = AGENTS * el * (K_PR / k_s)
    return {"value": 1.0 / step_s, "unit": "control_steps/s", "cores": threads, "kind": kind,
            "sample": f"1 agent: PR rollout of {k_s} samples x {P_PR} hypotheses x 2 plans x {H} steps, {reps} repetitions "
                      f"({time.perf_counter() - t0:.1f} s), scaled to 4 agents x K={K_PR}",
            "ms_per_control_step": step_s * 1e3}


def run_ours_pr(args) -> None:
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    drb = _package()
    import drone_race_b200.controllers as ctl_mod

    abi = drb.abi
    scs = _pr_workload(rank)
    stream = torch.cuda.Stream()
    ctls = [ctl_mod.PRMPPIController(s.env, s.prmppi, s.seed, device=local, stream=stream.cuda_stream) for s in scs]
    batch = ctl_mod.PRMPPIBatch(ctls, stream=stream.cuda_stream)
    if args.pr_slots is not None:
        batch.set_rollout_slots(args.pr_slots)
    n = len(ctls)
    states = [s.state for s in scs]
    beliefs = np.stack([s.belief() for s in scs])
    st_dev = torch.frombuffer(bytearray(bytes((abi.dr_sim_state * n)(*states))), dtype=torch.uint8).to("cuda")
    bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
    bel[:, :NTH_PR] = beliefs
    bel_dev = torch.from_numpy(bel).to("cuda")
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        batch.step_dev(st_dev.data_ptr(), bel_dev.data_ptr())
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.step_dev(st_dev.data_ptr(), bel_dev.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    _barrier(world)
    ms = _max_over_ranks(e0.elapsed_time(e1), world)
    # per-kernel times: a pass after the timed region with CUDA events between the kernels
    batch.set_profiling(True)
    for _ in range(args.steps):
        batch.step_dev(st_dev.data_ptr(), bel_dev.data_ptr())
    torch.cuda.synchronize()
    kt = batch.kernel_times()
    batch.set_profiling(False)
    ms_per_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    for c in ctls:
        c.engine = object()
    e2e_steps = 0 if args.quick else args.steps
    for _ in range(0 if args.quick else args.warmup):
        batch.step(states, beliefs)
    torch.cuda.synchronize()
    _barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        batch.step(states, beliefs)
    t1 = time.perf_counter()
    _barrier(world)
    e2e_s = _max_over_ranks(max(t1 - t0, 1e-9), world)
    h2d = d2h = 0
    for c in ctls:
        a, b = C.c_size_t(), C.c_size_t()
        abi.lib().dr_prmppi_io_bytes(c.handle, C.byref(a), C.byref(b))
        h2d += a.value
        d2h += b.value
    units = AGENTS * 2 * P_PR * K_PR * H
    dom = max(kt, key=kt.get) if kt else None
    roof = None
    if dom and "rollout" in dom and clk.get("sm_mhz"):
        peak = 2 * 128 * 148 * clk["sm_mhz"] * 1e6 / 1e12
        achieved = units * PR_FLOPS_PER_ROLLOUT_STEP / (kt[dom] / 1e3) / 1e12
        roof = {"bound": "fp32", "kernel": f"pr_{dom}" if not dom.startswith("pr") else dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "FP32 FMA rate of 148 SMs x 128 lanes at the median SM clock sampled during the timed region (MEASURED_PEAKS.json has no FP32 figure)",
                "units_per_launch": units, "flops_per_unit": PR_FLOPS_PER_ROLLOUT_STEP, "kernel_ms": kt[dom],
                "measured": "CUDA events around each launch on its stream over the timed region"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.quick:
        cpu = cpu_baseline_pr(scs)
        cpu.pop("ms_per_control_step", None)
    line = {
        "metric": "control_steps_per_s",
        "value": value,
        "unit": _unit(),
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded tracks, hypotheses and beliefs; no dataset)",
        "config": {"workload": _workload_name(), "agents": AGENTS, "K": K_PR, "H": H, "P": P_PR, "n_theta": NTH_PR, "n_opp": 1,
                   "parallelism": f"replicas x{world}", "l2": "working set per step < L2; steps are dependent control steps of the same controllers"},
        "rollout_steps_per_s": world * units * args.steps / (ms / 1e3),
        "kernel_ms": kt,
        "e2e": None if args.quick else {"value": world * args.steps / e2e_s, "unit": "control steps/s", "h2d_bytes_per_step": h2d,
                                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s / args.steps * 1e3},
        "gpu_launches": len(kt) * args.steps,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    for c in ctls:
        c.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_reference_pr(args) -> None:
    """Reference arm of --workload pr: the reference's CPU PR rollout (host threads), and
    on a GPU box its own PRMPPIController::getControl on the same 4 agents."""
    scs = _pr_workload(0)
    ms = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline_pr(scs, target_s=min(20.0, 120.0 / max(1, args.warmup + args.steps)), max_reps=1)
        if i >= args.warmup:
            ms.append(r["ms_per_control_step"])
        base = r
    v = 1e3 / statistics.mean(ms)
    ref_cuda = None
    try:
        import torch

        if torch.cuda.is_available() and not args.no_reference_cuda:
            sys.path.insert(0, str(ROOT))
            from oracle import oracle as O

            drb = _package()
            O.set_abi(drb.abi)
            variant = O.ref_variant_name(NTH_PR, True)
            if O.ref_available(variant):
                out = (C.c_double * 2)()
                sc = scs[0]
                rc = O.ref(variant).refc_prmppi_time(C.byref(sc.env), C.byref(sc.prmppi), C.byref(sc.state), AGENTS, 3, 20, out)
                ref_cuda = ({"getcontrol_ms_per_step": out[0], "control_steps_per_s": 1e3 / out[0], "steps": 20, "warmup": 3,
                             "what": "reference PRMPPIController::getControl per agent, wall clock, compiled from its sources"}
                            if rc == 0 else {"error": f"reference CUDA timing failed with status {rc}"})
    except Exception as e:  # measurement only
        ref_cuda = {"error": repr(e)}
    print(json.dumps({"impl": "reference", "metric": "control_steps_per_s", "value": v, "unit": _unit(), "n_gpus": 1, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic (seeded tracks, hypotheses and beliefs; no dataset)",
                      "config": {"workload": _workload_name(), "agents": AGENTS, "K": K_PR, "H": H, "P": P_PR, "n_theta": NTH_PR,
                                 "parallelism": "host threads"},
                      "cpu_baseline": {"value": v, "unit": "control_steps/s", "cores": base["cores"], "kind": base["kind"], "sample": base["sample"]},
                      "e2e": {"value": v, "unit": "control steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                      "reference_cuda": ref_cuda}), flush=True)


def run_ours_races(args) -> None:
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    drb = _package()
    import drone_race_b200.controllers as ctl_mod

    abi = drb.abi
    scs = drb.scenarios.uneven_races(N_RACES, seed=rank, n_verif=V_RACES)
    groups = [g for g in ([s for s in scs if not s.mppi.use_splines], [s for s in scs if s.mppi.use_splines]) if g]
    runs = []
    for g in groups:
        stream = torch.cuda.Stream()
        ctls = [ctl_mod.MPPIController(s.env, s.mppi, s.seed, device=local, stream=stream.cuda_stream) for s in g]
        batch = ctl_mod.MPPIBatch(ctls, stream=stream.cuda_stream)
        n = len(g)
        states = [s.state for s in g]
        st_dev = torch.frombuffer(bytearray(bytes((type(states[0]) * n)(*states))), dtype=torch.uint8).to("cuda")
        bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
        bel[:, :N_THETA] = np.stack([s.belief() for s in g])
        runs.append({"stream": stream, "ctls": ctls, "batch": batch, "scs": g, "st": st_dev, "bel": torch.from_numpy(bel).to("cuda"),
                     "act": torch.zeros((n, 2), dtype=torch.float32, device="cuda"),
                     "info": torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")})
    torch.cuda.synchronize()
    n_agents = len(scs)

    def dev_step():
        for r in runs:
            r["batch"].step_device(r["st"].data_ptr(), r["bel"].data_ptr(), r["act"].data_ptr(), r["info"].data_ptr())

    def timed(steps: int):
        for _ in range(args.warmup):
            dev_step()
        torch.cuda.synchronize()
        _barrier(world)
        s0 = runs[0]["stream"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        for r in runs[1:]:
            r["stream"].wait_event(e0)
        for _ in range(steps):
            dev_step()
        for r in runs[1:]:
            ev = torch.cuda.Event()
            ev.record(r["stream"])
            s0.wait_event(ev)
        e1.record(s0)
        torch.cuda.synchronize()
        _barrier(world)
        return _max_over_ranks(e0.elapsed_time(e1), world)

    # The controllers' plans keep changing from step to step (and with them how long the
    # rollouts run before they end), so the launch shapes are timed in interleaved rounds
    # after a longer warm-up, each shape for a third of the steps per round.
    for _ in range(10):
        dev_step()
    torch.cuda.synchronize()
    fixed = (("one_cta_per_tile", (0, 0, 0)), ("persistent_queue", (-1, -1, 0)), ("one_cta_per_tile_lockstep", (0, 0, 1)))
    tune = [r["batch"].autotune(5) for r in runs]
    tuned = [(t["rollout_ctas_per_sm"], t["verify_ctas_per_sm"], t["rollout_lockstep"]) for t in tune]
    per_round = max(1, args.steps // 3)
    totals = {name: 0.0 for name, _ in fixed}
    totals["autotuned"] = 0.0
    clocks = Clocks(local)
    clocks.start()
    for _ in range(3):
        for name, shape in fixed + (("autotuned", None),):
            for r, tshape in zip(runs, tuned):
                r["batch"].set_persistent(*(shape if shape is not None else tshape))
            totals[name] += timed(per_round)
    clk = clocks.stop()
    n_timed = 3 * per_round
    shapes = {name: {"ms_per_step": totals[name] / n_timed} for name, _ in fixed}
    ms = totals["autotuned"] * args.steps / n_timed
    shapes["autotuned"] = {"ms_per_step": ms / args.steps,
                           "choices": [{k: t[k] for k in ("rollout_ctas_per_sm", "rollout_lockstep", "verify_ctas_per_sm")} for t in tune],
                           "candidates_ms": [{"rollout": {f"{c}x{l}": v for (c, l), v in t["rollout"].items()}, "verify": t["verify"]} for t in tune]}
    for v in shapes.values():
        v["agent_control_steps_per_s"] = world * n_agents / (v["ms_per_step"] / 1e3)
    ms_per_step = ms / args.steps
    # per-kernel device times with the tuned shapes
    for r in runs:
        r["batch"].set_profiling(True)
    for _ in range(max(3, min(10, args.steps))):
        dev_step()
    torch.cuda.synchronize()
    kts = [r["batch"].kernel_times() for r in runs]
    for r in runs:
        r["batch"].set_profiling(False)
    # end to end through the C ABI with host buffers (both batches, one after the other)
    e2e = None
    if not args.quick:
        for r in runs:
            for c in r["ctls"]:
                c.engine = object()
        host = [([s.state for s in r["scs"]], np.stack([s.belief() for s in r["scs"]])) for r in runs]
        for _ in range(2):
            for r, (st, be) in zip(runs, host):
                r["batch"].step(st, be)
        torch.cuda.synchronize()
        e2e_steps = max(3, min(20, args.steps))
        _barrier(world)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for r, (st, be) in zip(runs, host):
                r["batch"].step(st, be)
        t1 = time.perf_counter()
        _barrier(world)
        e2e_s = _max_over_ranks(t1 - t0, world)
        h2d = d2h = 0
        for r in runs:
            for c in r["ctls"]:
                a, b = C.c_size_t(), C.c_size_t()
                abi.lib().dr_mppi_io_bytes(c.handle, C.byref(a), C.byref(b))
                h2d += a.value
                d2h += b.value
        e2e = {"value": world * n_agents * e2e_steps / e2e_s, "unit": "agent control steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_s / e2e_steps * 1e3}
    rollout_units = sum(s.mppi.n_samples * N_THETA * s.mppi.n_timesteps for s in scs)
    verify_units = sum(2 * V_RACES * min(40, s.mppi.n_timesteps) for s in scs)
    kt_sum = {}
    for kt in kts:
        for k, v in kt.items():
            kt_sum[k] = kt_sum.get(k, 0.0) + v
    roof = None
    if clk.get("sm_mhz"):
        peak = 2 * 128 * 148 * clk["sm_mhz"] * 1e6 / 1e12
        ach = (rollout_units * FLOPS_PER_ROLLOUT_STEP + verify_units * FLOPS_PER_VERIFY_STEP) / (ms_per_step / 1e3) / 1e12
        roof = {"bound": "fp32", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
                "scope": "all FP32 work of one control step of every agent (dense-control FLOP counts; spline evaluation not counted) / device step time",
                "peak_source": "FP32 FMA rate of 148 SMs x 128 lanes at the median SM clock sampled during the timed region"}
    line = {
        "metric": "agent_control_steps_per_s",
        "value": shapes["autotuned"]["agent_control_steps_per_s"],
        "unit": f"agent control steps/s ({N_RACES} races, {n_agents} agents of uneven K/H, every agent advanced once per step)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uneven races; no dataset)",
        "config": {"workload": f"uneven_races_{N_RACES}", "agents": n_agents, "K_total": sum(s.mppi.n_samples for s in scs),
                   "H": sorted({s.mppi.n_timesteps for s in scs}), "verif_samples": V_RACES, "batches": len(runs), "parallelism": f"replicas x{world}",
                   "l2": "working set per step > L2 (costs and plans of all agents)"},
        "shapes": shapes,
        "rollout_steps_per_s": world * rollout_units / (ms_per_step / 1e3),
        "kernel_ms": kt_sum,
        "e2e": e2e,
        "gpu_launches": sum(len(kt) for kt in kts) * args.steps,
        "roofline": roof,
        "cpu_baseline": None,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for r in runs:
        r["batch"].close()
        for c in r["ctls"]:
            c.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_ours_mixed(args) -> None:
    """--workload races: the batched uneven workload of mixed controller kinds
    (scenarios.mixed_races: 256 races of U{1..8} agents, plain MPPI, gradient-refined MPPI
    and PR-MPPI with B in {2, 4, 8}). Controllers of one kind and compile-time shape share a
    batch (MPPI: plain and gradient-refined together, one batch per control mode; PR-MPPI:
    one batch per B), each batch on its own stream, all stepped from device-resident inputs;
    one control step = every agent of every race advanced once. Reported: aggregate agent
    control steps/s and rollout-steps/s (steps pipelined), and the per-agent control-step
    latency (p50 / p99 over agents x steps of the time from a step's start, all batches
    launched together, to the end of the agent's batch)."""
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    drb = _package()
    import drone_race_b200.controllers as ctl_mod

    abi = drb.abi
    scs = drb.scenarios.mixed_races(N_RACES, seed=rank, n_verif=V_RACES)
    groups = []
    for spl in (False, True):
        g = [s for s in scs if s.kind in ("plain", "grad") and bool(s.mppi.use_splines) == spl]
        if g:
            groups.append(("mppi", g))
    for B in (2, 4, 8):
        g = [s for s in scs if s.kind == "pr" and s.n_theta == B]
        if g:
            groups.append(("pr", g))
    runs = []
    for kind, g in groups:
        stream = torch.cuda.Stream()
        n = len(g)
        states = [s.state for s in g]
        st_dev = torch.frombuffer(bytearray(bytes((type(states[0]) * n)(*states))), dtype=torch.uint8).to("cuda")
        bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
        for i, s in enumerate(g):
            bel[i, : s.n_theta] = s.belief()
        r = {"kind": kind, "stream": stream, "scs": g, "st": st_dev, "bel": torch.from_numpy(bel).to("cuda")}
        if kind == "mppi":
            ctls = [ctl_mod.MPPIController(s.env, s.mppi, s.seed, device=local, stream=stream.cuda_stream) for s in g]
            for c, s in zip(ctls, g):
                if s.kind == "grad":
                    c.set_grad_refine(GRAD_STEPS, GRAD_STEP_SIZE, 0)
            r["batch"] = ctl_mod.MPPIBatch(ctls, stream=stream.cuda_stream)
            r["act"] = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
            r["info"] = torch.zeros(C.sizeof(abi.dr_mppi_info) * n, dtype=torch.uint8, device="cuda")
        else:
            ctls = [ctl_mod.PRMPPIController(s.env, s.prmppi, s.seed, device=local, stream=stream.cuda_stream) for s in g]
            r["batch"] = ctl_mod.PRMPPIBatch(ctls, stream=stream.cuda_stream)
            if args.pr_slots is not None:
                r["batch"].set_rollout_slots(args.pr_slots)
        r["ctls"] = ctls
        runs.append(r)
    torch.cuda.synchronize()
    n_agents = len(scs)

    def run_step(r):
        if r["kind"] == "mppi":
            r["batch"].step_device(r["st"].data_ptr(), r["bel"].data_ptr(), r["act"].data_ptr(), r["info"].data_ptr())
        else:
            r["batch"].step_dev(r["st"].data_ptr(), r["bel"].data_ptr())

    def dev_step():
        for r in runs:
            run_step(r)

    s0 = runs[0]["stream"]

    def timed(steps: int) -> float:
        torch.cuda.synchronize()
        _barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        for r in runs[1:]:
            r["stream"].wait_event(e0)
        for _ in range(steps):
            dev_step()
        for r in runs[1:]:
            ev = torch.cuda.Event()
            ev.record(r["stream"])
            s0.wait_event(ev)
        e1.record(s0)
        torch.cuda.synchronize()
        _barrier(world)
        return _max_over_ranks(e0.elapsed_time(e1), world)

    for _ in range(10):
        dev_step()
    torch.cuda.synchronize()
    tune = [r["batch"].autotune(5) if r["kind"] == "mppi" else None for r in runs]
    for _ in range(max(args.warmup, 3)):
        dev_step()
    clocks = Clocks(local)
    clocks.start()
    ms = timed(args.steps)
    clk = clocks.stop()
    ms_per_step = ms / args.steps
    # per-step latency: each step starts when the previous one has ended everywhere
    lat_steps = max(5, min(30, args.steps))
    marks = []
    torch.cuda.synchronize()
    for _ in range(lat_steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        ends = []
        for r in runs:
            r["stream"].wait_event(e0)
            run_step(r)
            e = torch.cuda.Event(enable_timing=True)
            e.record(r["stream"])
            ends.append(e)
        for e in ends:
            s0.wait_event(e)
        marks.append((e0, ends))
    torch.cuda.synchronize()
    per_agent = []
    step_ms = []
    for e0, ends in marks:
        t = [e0.elapsed_time(e) for e in ends]
        step_ms.append(max(t))
        for r, tr in zip(runs, t):
            per_agent += [tr] * len(r["scs"])
    per_agent = np.array(per_agent)
    latency = {"p50_ms": float(np.percentile(per_agent, 50)), "p99_ms": float(np.percentile(per_agent, 99)), "max_ms": float(per_agent.max()),
               "step_ms_median": float(np.median(step_ms)), "samples": int(per_agent.size),
               "what": "per agent and step: from the step's start (all batches launched together) to the end of the agent's batch"}
    # per-kernel device times
    for r in runs:
        r["batch"].set_profiling(True)
    for _ in range(3):
        dev_step()
    torch.cuda.synchronize()
    kts = [r["batch"].kernel_times() for r in runs]
    for r in runs:
        r["batch"].set_profiling(False)
    # end to end through the C ABI with host buffers, one batch after the other
    e2e = None
    if not args.quick:
        for r in runs:
            for c in r["ctls"]:
                c.engine = object()
        host = [([s.state for s in r["scs"]], np.stack([s.belief() for s in r["scs"]])) for r in runs]
        for _ in range(2):
            for r, (st, be) in zip(runs, host):
                r["batch"].step(st, be)
        torch.cuda.synchronize()
        e2e_steps = max(3, min(10, args.steps))
        _barrier(world)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for r, (st, be) in zip(runs, host):
                r["batch"].step(st, be)
        t1 = time.perf_counter()
        _barrier(world)
        e2e_s = _max_over_ranks(t1 - t0, world)
        h2d = d2h = 0
        for r in runs:
            fn = abi.lib().dr_mppi_io_bytes if r["kind"] == "mppi" else abi.lib().dr_prmppi_io_bytes
            for c in r["ctls"]:
                a, b = C.c_size_t(), C.c_size_t()
                fn(c.handle, C.byref(a), C.byref(b))
                h2d += a.value
                d2h += b.value
        e2e = {"value": world * n_agents * e2e_steps / e2e_s, "unit": "agent control steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_s / e2e_steps * 1e3}
    mppi_scs = [s for s in scs if s.kind != "pr"]
    pr_scs = [s for s in scs if s.kind == "pr"]
    rollout_units = sum(s.mppi.n_samples * s.n_theta * s.mppi.n_timesteps for s in mppi_scs)
    verify_units = sum(2 * V_RACES * min(40, s.mppi.n_timesteps) for s in mppi_scs)
    pr_units = sum(2 * s.prmppi.P * s.prmppi.n_samples * s.prmppi.n_timesteps for s in pr_scs)
    roof = None
    if clk.get("sm_mhz"):
        peak = 2 * 128 * 148 * clk["sm_mhz"] * 1e6 / 1e12
        ach = (rollout_units * FLOPS_PER_ROLLOUT_STEP + verify_units * FLOPS_PER_VERIFY_STEP + pr_units * PR_FLOPS_PER_ROLLOUT_STEP) / (ms_per_step / 1e3) / 1e12
        roof = {"bound": "fp32", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
                "scope": "FP32 work of the MPPI rollouts and verifications and the PR-MPPI rollouts of one control step of every agent (dense-control "
                         "FLOP counts; spline evaluation, updates, gradient refinement and candidate re-checks not counted) / device step time",
                "peak_source": "FP32 FMA rate of 148 SMs x 128 lanes at the median SM clock sampled during the timed region"}
    kinds = {k: sum(1 for s in scs if s.kind == k) for k in ("plain", "grad", "pr")}
    line = {
        "metric": "agent_control_steps_per_s",
        "value": world * n_agents / (ms_per_step / 1e3),
        "unit": f"agent control steps/s ({N_RACES} races, {n_agents} agents of uneven K/H and mixed kinds, every agent advanced once per step)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uneven races of mixed controller kinds; no dataset)",
        "config": {"workload": f"mixed_races_{N_RACES}", "agents": n_agents, "kinds": kinds,
                   "pr_branches": {str(B): sum(1 for s in pr_scs if s.n_theta == B) for B in (2, 4, 8)},
                   "K_total": sum(s.mppi.n_samples if s.mppi else s.prmppi.n_samples for s in scs),
                   "H": sorted({(s.mppi or s.prmppi).n_timesteps for s in scs}), "verif_samples": V_RACES, "grad_steps": GRAD_STEPS,
                   "batches": [f"{r['kind']}:{len(r['scs'])}" for r in runs], "parallelism": f"replicas x{world}",
                   "l2": "working set per step > L2 (costs and plans of all agents)"},
        "latency": latency,
        "rollout_steps_per_s": world * (rollout_units + pr_units) / (ms_per_step / 1e3),
        "kernel_ms": kts,
        "autotune": [None if t is None else {k: t[k] for k in ("rollout_ctas_per_sm", "rollout_lockstep", "verify_ctas_per_sm", "grad_ckpt")} for t in tune],
        "e2e": e2e,
        "gpu_launches": sum(len(kt) for kt in kts) * args.steps,
        "roofline": roof,
        "cpu_baseline": None,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for r in runs:
        r["batch"].close()
        for c in r["ctls"]:
            c.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def reference_cpu_step(scs, variant: str, threads: int, noises) -> float:
    """One control step of the 4-agent workload on the reference's own CPU path (its
    model functions in host loops, oracle/_ref, OpenMP over `threads`): per agent the
    full K-sample rollout, the update (aggregation, masked minima, weighted averages,
    clamp), and the verification of the new and the previous plan over V samples x the
    verification horizon. Returns the seconds it took."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    for sc, noise in zip(scs, noises):
        belief = sc.belief()
        prev = np.zeros((N_THETA + 1, H, 2), np.float32)
        ct, bu, bt = O.mppi_rollout(sc, belief, prev, noise, None, 0, impl=variant, nthreads=threads)
        _, dense, _, _, _ = O.mppi_update(sc, belief, ct, bu, bt, noise, None, prev, impl=variant, nthreads=threads)
        O.mppi_verify(sc, belief, dense, 0, 0, impl=variant, nthreads=threads)
        O.mppi_verify(sc, belief, prev, 0, 1, impl=variant, nthreads=threads)
    return time.perf_counter() - t0


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if WL["kind"] in ("races", "races_mppi"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference steps one controller per getControl call and has no multi-race batch; "
                                                              "its per-controller rate is the strat and pr workloads' reference arm"}), flush=True)
        return
    if WL["kind"] == "grad":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no gradient-refined MPPI; its plain MPPI arm is --workload strat"}),
              flush=True)
        return
    if WL["kind"] == "pr":
        run_reference_pr(args)
        return
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O

    drb = _package()
    O.set_abi(drb.abi)
    scs = workload(0)
    variant = _ref_variant(O)
    if not O.ref_available(variant):
        print(json.dumps({"impl": "reference", "unavailable": f"the reference build oracle/_ref/libref_{variant}.so is missing (make -C oracle ref)"}),
              flush=True)
        return
    threads = os.cpu_count() or 1
    # the perturbations the reference's generateNoiseKernel would draw, made once before
    # the timed steps (the CPU path has no noise kernel of its own)
    noises = [O.mppi_noise(sc, 0) for sc in scs]
    steps_s = []
    for i in range(args.warmup + args.steps):
        dt = reference_cpu_step(scs, variant, threads, noises)
        if i >= args.warmup:
            steps_s.append(dt)
    ms = statistics.mean(steps_s) * 1e3
    value = 1e3 / ms
    sample = (f"the whole workload every step, no scaling: {AGENTS} agents x (rollout of K={_K()} samples x {N_THETA} hypotheses x {H} steps, "
              f"update, verification of 2 plans x V={V} samples x {VERIF_H} steps); perturbations precomputed")
    line = {
        "impl": "reference",
        "metric": "control_steps_per_s",
        "value": value,
        "unit": _unit(),
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded tracks and states; no dataset)",
        "config": {"workload": _workload_name(), "agents": AGENTS, "K": _K(), "H": H, "n_theta": N_THETA, "n_opp": 1, "controls": "dense",
                   "verif_samples": V, "verif_horizon": VERIF_H, "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": value, "unit": "control_steps/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "control steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": None if args.no_reference_cuda else reference_cuda_timing(scs),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (no e2e, no CPU baseline): for profiler runs")
    ap.add_argument("--no-overlap", action="store_true", help="run the previous plan's verification after the rollout instead of beside it")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="strat", choices=["strat", "gates", "grad", "pr", "races", "races_mppi"],
                    help="strat: the strategic race (the headline workload); gates: the gate race (EnvDroneRace); "
                         "grad: gradient-refined MPPI at K=1024 with a closed-loop comparison against plain MPPI at K=4096; "
                         "pr: PR-MPPI, 4 agents x 8 hypotheses x K=2048; "
                         "races: 256 independent races of uneven K/H and mixed kinds (plain, gradient-refined and PR-MPPI); "
                         "races_mppi: the same races with plain MPPI only, one batch per control mode")
    ap.add_argument("--side-verify", type=int, default=None,
                    help="CTAs per SM of the previous plan's verification beside the rollout (0: one per tile; default: the library's)")
    ap.add_argument("--pdl", action="store_true", help="programmatic dependent launches of the update and the new plan's verification")
    ap.add_argument("--pr-slots", type=int, default=None, choices=[1, 2, 4],
                    help="pr and races workloads: hypothesis slots per PR-MPPI rollout thread sharing the ego's moves (default: the library's)")
    ap.add_argument("--grad-steps", type=int, default=GRAD_STEPS, help="grad workload: projected gradient steps after each update")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true", help="reference arm: skip timing the reference's CUDA path")
    args = ap.parse_args()
    globals()["GRAD_STEPS"] = args.grad_steps
    WL["kind"] = args.workload
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif WL["kind"] == "pr":
        run_ours_pr(args)
    elif WL["kind"] == "races":
        run_ours_mixed(args)
    elif WL["kind"] == "races_mppi":
        run_ours_races(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
