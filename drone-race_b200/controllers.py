"""Controller classes over the C ABI, mirroring the reference's controller interface
(include/controllers.h:12-179): `getControl(state) -> action`, with the public fields
the reference's simulation engine reads after each call (src/engine.cpp:73-212).

All compute happens in lib/libdrmppi.so; these classes only marshal arguments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import check, lib


def _state(s, gate: bool = False):
    want = abi.dr_gate_state if gate else abi.dr_sim_state
    if isinstance(s, want):
        return s
    raise TypeError(f"state must be a {want.__name__}")


def _predict(call, rows: int, T: int, n_agents: int, what: str) -> dict:
    """Runs a prediction entry point into fresh host arrays (layout of include/drmppi.h)."""
    pos = np.zeros((rows, T, n_agents * 2), np.float32)
    act = np.zeros((rows, T, 2), np.float32)
    rec = np.zeros((rows, abi.DR_PREDICT_RECORD), np.int32)
    cost = np.zeros(rows, np.float32)
    check(call(pos, act, rec, cost), what)
    return dict(positions=pos, actions=act, init_branch=rec[:, 0].copy(), branching_time=rec[:, 1].copy(), branch=rec[:, 2].copy(),
                stop_reason=rec[:, 3].copy(), stop_time=rec[:, 4].copy(), cost=cost)


class Controller:
    """include/controllers.h:12-21."""

    def __init__(self, n_theta: int, init_belief: np.ndarray):
        self.engine = None
        self.h_belief = np.array(init_belief[:n_theta], dtype=np.float32)

    def getControl(self, state) -> np.ndarray:  # noqa: N802 (reference name)
        raise NotImplementedError


class MPPIController(Controller):
    """MPPIController (include/controllers.h:23-111, src/mppi_controller.cu). `env` is a
    dr_env_config (the strategic race) or a dr_gate_env_config (the gate race, the
    reference's controller compiled with USE_ENV_DRONERACE); states match it."""

    def __init__(self, env, cfg: abi.dr_mppi_config, seed: int, nominal: np.ndarray | None = None, device: int = 0, stream=None):
        super().__init__(env.n_theta, np.array(env.init_belief))
        self.mppiConfig = cfg
        self.n_theta = int(env.n_theta)
        self.T = int(cfg.n_timesteps)
        self.nbp = self.n_theta + 1
        h = C.c_void_p()
        nom = None
        if nominal is not None:
            nominal = np.ascontiguousarray(nominal, np.float32)
            if nominal.size != self.nbp * self.T * 2:
                raise ValueError(f"Invalid MPPI construction: expected nominal size {self.nbp * self.T * 2}, got {nominal.size}")
            nom = abi.fptr(nominal)
        self.gate = isinstance(env, abi.dr_gate_env_config)
        self.n_agents = 2 if self.gate else int(env.n_opp) + 1
        create = lib().dr_gate_mppi_create if self.gate else lib().dr_mppi_create
        check(create(C.byref(env), C.byref(cfg), seed, nom, device, C.c_void_p(stream) if stream else None, C.byref(h)), "dr_mppi_create")
        self._h = h
        self.info = abi.dr_mppi_info()
        self.failCount = np.zeros(self.T, np.uint32)
        self.failCountNew = np.zeros(self.T, np.uint32)
        self.failCountOld = np.zeros(self.T, np.uint32)
        self.min_nu = float(cfg.min_nu) or 0.0005
        self.max_nu = float(cfg.max_nu) or 0.001

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def predict(self, state, belief) -> dict:
        """The engine's prediction streaming for this controller (dr_mppi_predict): from the
        state after the step, under every hypothesis, the plan the controller holds."""
        bel = np.ascontiguousarray(belief, np.float32)
        return _predict(lambda pos, act, rec, cost: lib().dr_mppi_predict(self._h, C.byref(state), abi.fptr(bel), abi.fptr(pos), abi.fptr(act),
                                                                         abi.iptr(rec), abi.fptr(cost)),
                        self.n_theta, self.T, self.n_agents, "dr_mppi_predict")

    def set_verify_exact(self, on: bool = True) -> None:
        """Verification flavour (dr_mppi_set_verify_exact): exact reproduces the CPU
        oracle's per-sample results; the default fast flavour agrees in distribution."""
        check(lib().dr_mppi_set_verify_exact(self._h, int(bool(on))), "dr_mppi_set_verify_exact")

    def set_ego_table(self, on: bool = True) -> None:
        """Whether the fast verification reads the ego from the shared ego tables
        (dr_mppi_set_ego_table; the default) or moves it in every sample."""
        check(lib().dr_mppi_set_ego_table(self._h, int(bool(on))), "dr_mppi_set_ego_table")

    def close(self) -> None:
        if self._h:
            lib().dr_mppi_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getControl(self, state) -> np.ndarray:  # noqa: N802
        if self.engine is None:
            raise RuntimeError("MPPI: engine not set")
        out = np.zeros(2, np.float32)
        step = lib().dr_gate_mppi_step if self.gate else lib().dr_mppi_step
        check(step(self._h, C.byref(_state(state, self.gate)), abi.fptr(self.h_belief), abi.fptr(out), C.byref(self.info)), "dr_mppi_step")
        self._pull()
        return out

    def _pull(self) -> None:
        check(lib().dr_mppi_get_fail_counts(self._h, abi.uptr(self.failCountNew), abi.uptr(self.failCountOld), abi.uptr(self.failCount), self.T),
              "dr_mppi_get_fail_counts")

    # public fields of the reference controller
    @property
    def h_nominal(self) -> np.ndarray:
        out = np.zeros(self.nbp * self.T * 2, np.float32)
        check(lib().dr_mppi_get_nominal(self._h, abi.fptr(out), out.size), "dr_mppi_get_nominal")
        return out

    def set_grad_refine(self, steps: int, step_size: float = 0.05, ckpt_stride: int = 0) -> None:
        """Gradient-refined MPPI: `steps` projected gradient steps on the noise-free
        rollout objective after each update, the best of the plain update and the
        iterates kept (dr_mppi_set_grad_refine). Strategic race only; call it before
        batching this controller."""
        check(lib().dr_mppi_set_grad_refine(self._h, int(steps), float(step_size), int(ckpt_stride)), "dr_mppi_set_grad_refine")

    def knots(self) -> np.ndarray:
        M = int(self.mppiConfig.n_knots) if self.mppiConfig.use_splines else self.T
        out = np.zeros(self.nbp * M * 2, np.float32)
        check(lib().dr_mppi_get_knots(self._h, abi.fptr(out), out.size), "dr_mppi_get_knots")
        return out.reshape(self.nbp, M, 2)

    @property
    def epsilon(self) -> float:
        return self.info.epsilon

    @property
    def epsilonPartial(self) -> float:  # noqa: N802
        return self.info.epsilon_partial

    @property
    def certifiedLoss(self) -> float:  # noqa: N802
        return self.info.certified_loss

    @property
    def useNewPlan(self) -> bool:  # noqa: N802
        return bool(self.info.use_new_plan)

    @property
    def invTemperature(self) -> float:  # noqa: N802
        return float(lib().dr_mppi_get_temperature(self._h))

    @property
    def step_index(self) -> int:
        return int(lib().dr_mppi_get_step(self._h))

    def set_profiling(self, on: bool) -> None:
        check(lib().dr_mppi_set_profiling(self._h, int(on)), "dr_mppi_set_profiling")

    def kernel_times(self) -> dict[str, float]:
        return _kernel_times(lib().dr_mppi_get_kernel_times, self._h)


class PRMPPIController(Controller):
    """PRMPPIController (include/controllers.h:114-179, src/prmppi_controller.cu)."""

    def __init__(self, env: abi.dr_env_config, cfg: abi.dr_prmppi_config, seed: int, nominal: np.ndarray | None = None, device: int = 0, stream=None):
        super().__init__(env.n_theta, np.array(env.init_belief))
        self.mppiConfig = cfg
        self.T = int(cfg.n_timesteps)
        h = C.c_void_p()
        nom = None
        if nominal is not None:
            nominal = np.ascontiguousarray(nominal, np.float32)
            if nominal.size != self.T * 2:
                raise ValueError(f"Invalid PRMPPI construction: expected nominal size {self.T * 2}, got {nominal.size}")
            nom = abi.fptr(nominal)
        self.gate = isinstance(env, abi.dr_gate_env_config)
        self.n_theta = int(env.n_theta)
        self.n_agents = 2 if self.gate else int(env.n_opp) + 1
        create = lib().dr_gate_prmppi_create if self.gate else lib().dr_prmppi_create
        check(create(C.byref(env), C.byref(cfg), seed, nom, device, C.c_void_p(stream) if stream else None, C.byref(h)), "dr_prmppi_create")
        self._h = h
        self.info = abi.dr_prmppi_info()
        self.min_nu = float(cfg.min_nu) or 0.0005
        self.max_nu = float(cfg.max_nu) or 0.001

    def predict(self, prev_state) -> dict:
        """The engine's prediction streaming for this controller (dr_prmppi_predict): from the
        state before the step, the new nominal plan under every hypothesis, then the robust
        plan under the last one."""
        return _predict(lambda pos, act, rec, cost: lib().dr_prmppi_predict(self._h, C.byref(prev_state), abi.fptr(pos), abi.fptr(act), abi.iptr(rec),
                                                                           abi.fptr(cost)),
                        self.n_theta + 1, self.T, self.n_agents, "dr_prmppi_predict")

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            lib().dr_prmppi_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getControl(self, state) -> np.ndarray:  # noqa: N802
        if self.engine is None:
            raise RuntimeError("PRMPPI: engine not set")
        out = np.zeros(2, np.float32)
        step = lib().dr_gate_prmppi_step if self.gate else lib().dr_prmppi_step
        check(step(self._h, C.byref(_state(state, self.gate)), abi.fptr(self.h_belief), abi.fptr(out), C.byref(self.info)), "dr_prmppi_step")
        return out

    def nominals(self) -> tuple[np.ndarray, np.ndarray]:
        a = np.zeros(self.T * 2, np.float32)
        b = np.zeros(self.T * 2, np.float32)
        check(lib().dr_prmppi_get_nominals(self._h, abi.fptr(a), abi.fptr(b), a.size), "dr_prmppi_get_nominals")
        return a, b

    @property
    def h_nom_nominal(self) -> np.ndarray:
        return self.nominals()[0]

    @property
    def h_rob_nominal(self) -> np.ndarray:
        return self.nominals()[1]

    @property
    def useNomPlan(self) -> bool:  # noqa: N802
        return bool(self.info.use_nom_plan)

    @property
    def resetNom(self) -> bool:  # noqa: N802
        return bool(self.info.reset_nom)

    def set_profiling(self, on: bool) -> None:
        check(lib().dr_prmppi_set_profiling(self._h, int(on)), "dr_prmppi_set_profiling")

    def kernel_times(self) -> dict[str, float]:
        return _kernel_times(lib().dr_prmppi_get_kernel_times, self._h)


def _kernel_times(fn, h) -> dict[str, float]:
    names = (C.c_char_p * 16)()
    ms = (C.c_float * 16)()
    cnt = C.c_int()
    check(fn(h, names, ms, 16, C.byref(cnt)), "get_kernel_times")
    return {names[i].decode(): float(ms[i]) for i in range(cnt.value)}


class _Sharded:
    """The exchange of a sample-sharded controller: its partial results gathered from
    every process of a torch.distributed group, on the controller's own stream (a torch
    stream handed to the library), so the library's kernels, the collectives and the next
    kernels run in order with no host synchronisation until the step's tail. With NCCL the
    tensors stay on the device; with gloo they travel through host memory."""

    def _setup(self, words: int, device: int, group):
        import torch

        self.group = group
        dev = torch.device("cuda", device)
        self._partial = torch.empty(words, dtype=torch.float32, device=dev)
        self._gathered = None
        self._words = words

    def _all_gather(self):
        import torch
        import torch.distributed as dist

        world = dist.get_world_size(self.group)
        with torch.cuda.stream(self._tstream):
            if self._gathered is None:
                self._gathered = torch.empty(world * self._words, dtype=torch.float32, device=self._partial.device)
            if dist.get_backend(self.group) == "gloo":
                parts = [torch.empty(self._words, dtype=torch.float32) for _ in range(world)]
                dist.all_gather(parts, self._partial.cpu(), group=self.group)
                self._gathered.copy_(torch.cat(parts))
            else:
                dist.all_gather_into_tensor(self._gathered, self._partial, group=self.group)
        return world

    def _all_reduce_sum(self, t):
        import torch
        import torch.distributed as dist

        with torch.cuda.stream(self._tstream):
            if dist.get_backend(self.group) == "gloo":
                x = t.cpu()
                dist.all_reduce(x, op=dist.ReduceOp.SUM, group=self.group)
                t.copy_(x)
            else:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)


class ShardedMPPIController(_Sharded, MPPIController):
    """One MPPI controller whose samples are split across the processes of a
    torch.distributed group (one process per GPU): this process rolls out and verifies its
    share; one all-gather of the partial minima, weighted sums and previous-plan failure
    histograms and one all-reduce of the new plan's histograms per step
    (dr_mppi_set_shard / dr_mppi_shard_*)."""

    def __init__(self, env, cfg: abi.dr_mppi_config, seed: int, rank: int, world: int, group=None, nominal: np.ndarray | None = None,
                 device: int = 0):
        import torch

        self._tstream = torch.cuda.Stream(device=device)
        super().__init__(env, cfg, seed, nominal=nominal, device=device, stream=self._tstream.cuda_stream)
        check(lib().dr_mppi_set_shard(self._h, int(rank), int(world)), "dr_mppi_set_shard")
        n = C.c_size_t()
        check(lib().dr_mppi_shard_words(self._h, C.byref(n)), "dr_mppi_shard_words")
        self._setup(int(n.value), device, group)
        self._hist = torch.empty(self.T, dtype=torch.int32, device=torch.device("cuda", device))

    def getControl(self, state) -> np.ndarray:  # noqa: N802
        if self.engine is None:
            raise RuntimeError("MPPI: engine not set")
        P = lambda t: C.c_void_p(t.data_ptr())
        bel = abi.fptr(self.h_belief)
        st = C.byref(_state(state, False))
        check(lib().dr_mppi_shard_begin(self._h, st, bel, P(self._partial)), "dr_mppi_shard_begin")
        world = self._all_gather()
        check(lib().dr_mppi_shard_update(self._h, P(self._gathered), world, P(self._hist)), "dr_mppi_shard_update")
        self._all_reduce_sum(self._hist)
        out = np.zeros(2, np.float32)
        check(lib().dr_mppi_shard_finish(self._h, P(self._hist), bel, abi.fptr(out), C.byref(self.info)), "dr_mppi_shard_finish")
        self._pull()
        return out


class ShardedPRMPPIController(_Sharded, PRMPPIController):
    """One PR-MPPI controller whose samples are split across the processes of a
    torch.distributed group: this process rolls out its share of the samples under every
    hypothesis; one all-gather of the partial minima and weighted sums per step
    (dr_prmppi_set_shard / dr_prmppi_shard_*); the candidates' re-check runs on every
    process."""

    def __init__(self, env, cfg: abi.dr_prmppi_config, seed: int, rank: int, world: int, group=None, nominal: np.ndarray | None = None,
                 device: int = 0):
        import torch

        self._tstream = torch.cuda.Stream(device=device)
        super().__init__(env, cfg, seed, nominal=nominal, device=device, stream=self._tstream.cuda_stream)
        check(lib().dr_prmppi_set_shard(self._h, int(rank), int(world)), "dr_prmppi_set_shard")
        n = C.c_size_t()
        check(lib().dr_prmppi_shard_words(self._h, C.byref(n)), "dr_prmppi_shard_words")
        self._setup(int(n.value), device, group)

    def getControl(self, state) -> np.ndarray:  # noqa: N802
        if self.engine is None:
            raise RuntimeError("PRMPPI: engine not set")
        P = lambda t: C.c_void_p(t.data_ptr())
        check(lib().dr_prmppi_shard_begin(self._h, C.byref(_state(state)), abi.fptr(self.h_belief), P(self._partial)), "dr_prmppi_shard_begin")
        world = self._all_gather()
        out = np.zeros(2, np.float32)
        check(lib().dr_prmppi_shard_finish(self._h, P(self._gathered), world, abi.fptr(out), C.byref(self.info)), "dr_prmppi_shard_finish")
        return out

class MPPIBatch:
    """Several MPPI controllers (one per agent) advanced by one launch sequence."""

    def __init__(self, controllers: list[MPPIController], stream=None):
        self.ctls = controllers
        arr = (C.c_void_p * len(controllers))(*[c.handle.value for c in controllers])
        b = C.c_void_p()
        check(lib().dr_mppi_batch_create(arr, len(controllers), C.c_void_p(stream) if stream else None, C.byref(b)), "dr_mppi_batch_create")
        self._b = b
        self.infos = (abi.dr_mppi_info * len(controllers))()
        # per-call buffers, allocated once (the call sits in closed control loops)
        n = len(controllers)
        gate = controllers[0].gate
        self._st = ((abi.dr_gate_state if gate else abi.dr_sim_state) * n)()
        self._bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
        self._out = np.zeros((n, 2), np.float32)
        self._step = lib().dr_gate_mppi_batch_step if gate else lib().dr_mppi_batch_step
        self._args = (self._st, abi.fptr(self._bel), abi.fptr(self._out), self.infos)

    def step(self, states, beliefs: np.ndarray) -> np.ndarray:
        for i, s in enumerate(states):
            self._st[i] = s
        self._bel[:, : beliefs.shape[1]] = beliefs
        self._bel[:, beliefs.shape[1]:] = 0.0
        check(self._step(self._b, *self._args), "dr_mppi_batch_step")
        return self._out.copy()

    def set_graph(self, on: bool) -> None:
        check(lib().dr_mppi_batch_set_graph(self._b, int(on)), "dr_mppi_batch_set_graph")

    def set_overlap(self, on: bool) -> None:
        check(lib().dr_mppi_batch_set_overlap(self._b, int(on)), "dr_mppi_batch_set_overlap")

    def set_priority(self, on: bool) -> None:
        check(lib().dr_mppi_batch_set_priority(self._b, int(on)), "dr_mppi_batch_set_priority")

    def set_persistent(self, rollout_ctas_per_sm: int, verify_ctas_per_sm: int, rollout_lockstep: bool = False) -> None:
        """Launch shape of the rollout and the verification: 0 = one CTA per tile, n > 0 =
        a persistent launch of n CTAs per SM fed by a device work queue, -1 = as many as
        fit; rollout_lockstep = a barrier per step in the rollout (dr_mppi_batch_set_persistent)."""
        check(lib().dr_mppi_batch_set_persistent(self._b, int(rollout_ctas_per_sm), int(verify_ctas_per_sm), int(rollout_lockstep)),
              "dr_mppi_batch_set_persistent")

    def set_side_verify(self, ctas_per_sm: int) -> None:
        """Shape of the previous plan's verification beside the critical path: n > 0 a
        persistent grid of n CTAs per SM (default 1), 0 one CTA per tile
        (dr_mppi_batch_set_side_verify)."""
        check(lib().dr_mppi_batch_set_side_verify(self._b, int(ctas_per_sm)), "dr_mppi_batch_set_side_verify")

    def set_pdl(self, on: bool) -> None:
        """Programmatic dependent launch of the update and the new plan's verification
        (dr_mppi_batch_set_pdl)."""
        check(lib().dr_mppi_batch_set_pdl(self._b, int(on)), "dr_mppi_batch_set_pdl")

    def autotune(self, reps: int = 5) -> dict:
        """Times the batch's launch-shape candidates on its current inputs and keeps the
        fastest (dr_mppi_batch_autotune); returns what was measured and chosen."""
        r = abi.dr_tune_report()
        check(lib().dr_mppi_batch_autotune(self._b, int(reps), C.byref(r)), "dr_mppi_batch_autotune")
        return {
            "rollout_ctas_per_sm": r.rollout_ctas_per_sm,
            "rollout_lockstep": r.rollout_lockstep,
            "verify_ctas_per_sm": r.verify_ctas_per_sm,
            "grad_ckpt": r.grad_ckpt,
            "rollout": {(int(r.rollout_cand[i]), int(r.rollout_lock[i])): float(r.rollout_ms[i]) for i in range(r.n_rollout)},
            "verify": {int(r.verify_cand[i]): float(r.verify_ms[i]) for i in range(r.n_verify)},
            "grad": {int(r.grad_cand[i]): float(r.grad_ms[i]) for i in range(r.n_grad)},
        }

    def step_dev(self, states_dev_ptr: int, beliefs_dev_ptr: int) -> None:
        """The control step's kernels on device-resident inputs, without its tail
        (dr_mppi_batch_step_dev)."""
        check(lib().dr_mppi_batch_step_dev(self._b, C.c_void_p(states_dev_ptr), C.c_void_p(beliefs_dev_ptr)), "dr_mppi_batch_step_dev")

    def step_device(self, states_dev_ptr: int, beliefs_dev_ptr: int, actions_dev_ptr: int, infos_dev_ptr: int) -> None:
        """The whole control step on the device, tail included (dr_mppi_batch_step_device):
        n states / n x DR_MAX_THETA beliefs in, n x 2 actions and n dr_mppi_info out, all
        device pointers; returns without waiting."""
        check(lib().dr_mppi_batch_step_device(self._b, C.c_void_p(states_dev_ptr), C.c_void_p(beliefs_dev_ptr), C.c_void_p(actions_dev_ptr),
                                              C.c_void_p(infos_dev_ptr)), "dr_mppi_batch_step_device")

    def env_step_device(self, true_theta_dev_ptr: int, actions_dev_ptr: int, states_dev_ptr: int, beliefs_dev_ptr: int, update_belief: bool, seed: int,
                        terms_dev_ptr: int) -> None:
        """Every controller's race advanced by one true-dynamics step on the device
        (dr_mppi_batch_env_step_device)."""
        check(lib().dr_mppi_batch_env_step_device(self._b, C.c_void_p(true_theta_dev_ptr), C.c_void_p(actions_dev_ptr), C.c_void_p(states_dev_ptr),
                                                  C.c_void_p(beliefs_dev_ptr), int(update_belief), int(seed), C.c_void_p(terms_dev_ptr)),
              "dr_mppi_batch_env_step_device")

    def set_profiling(self, on: bool) -> None:
        check(lib().dr_mppi_batch_set_profiling(self._b, int(on)), "dr_mppi_batch_set_profiling")

    def kernel_times(self) -> dict[str, float]:
        return _kernel_times(lib().dr_mppi_batch_get_kernel_times, self._b)

    def kernel_timeline(self) -> dict[str, tuple[float, float]]:
        """(start, end) of each timed kernel in ms after the start of the step."""
        names = (C.c_char_p * 16)()
        st = (C.c_float * 16)()
        en = (C.c_float * 16)()
        cnt = C.c_int()
        check(lib().dr_mppi_batch_get_kernel_timeline(self._b, names, st, en, 16, C.byref(cnt)), "get_kernel_timeline")
        return {names[i].decode(): (float(st[i]), float(en[i])) for i in range(cnt.value)}

    def close(self) -> None:
        if self._b:
            lib().dr_mppi_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PRMPPIBatch:
    def __init__(self, controllers: list[PRMPPIController], stream=None):
        self.ctls = controllers
        arr = (C.c_void_p * len(controllers))(*[c.handle.value for c in controllers])
        b = C.c_void_p()
        check(lib().dr_prmppi_batch_create(arr, len(controllers), C.c_void_p(stream) if stream else None, C.byref(b)), "dr_prmppi_batch_create")
        self._b = b
        self.infos = (abi.dr_prmppi_info * len(controllers))()
        n = len(controllers)
        self._st = (abi.dr_sim_state * n)()
        self._bel = np.zeros((n, abi.DR_MAX_THETA), np.float32)
        self._out = np.zeros((n, 2), np.float32)
        self._args = (self._st, abi.fptr(self._bel), abi.fptr(self._out), self.infos)

    def step(self, states, beliefs: np.ndarray) -> np.ndarray:
        for i, s in enumerate(states):
            self._st[i] = s
        self._bel[:, : beliefs.shape[1]] = beliefs
        self._bel[:, beliefs.shape[1]:] = 0.0
        check(lib().dr_prmppi_batch_step(self._b, *self._args), "dr_prmppi_batch_step")
        return self._out.copy()

    def step_dev(self, states_dev_ptr: int, beliefs_dev_ptr: int) -> None:
        check(lib().dr_prmppi_batch_step_dev(self._b, C.c_void_p(states_dev_ptr), C.c_void_p(beliefs_dev_ptr)), "dr_prmppi_batch_step_dev")

    def set_rollout_slots(self, slots: int) -> None:
        """Hypothesis slots per rollout thread, sharing the ego's moves
        (dr_prmppi_batch_set_rollout_slots); bit-identical costs for every choice."""
        check(lib().dr_prmppi_batch_set_rollout_slots(self._b, int(slots)), "dr_prmppi_batch_set_rollout_slots")

    def set_profiling(self, on: bool) -> None:
        check(lib().dr_prmppi_batch_set_profiling(self._b, int(on)), "dr_prmppi_batch_set_profiling")

    def kernel_times(self) -> dict[str, float]:
        return _kernel_times(lib().dr_prmppi_batch_get_kernel_times, self._b)

    def close(self) -> None:
        if self._b:
            lib().dr_prmppi_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def env_step(env: abi.dr_env_config, true_theta: int, action, state: abi.dr_sim_state, belief: np.ndarray, update_belief: bool, seed: int,
             step: int) -> int:
    """One true-dynamics step on the device (engine dynStep, src/engine.cpp:286-312);
    state and belief are updated in place; returns the terminal type."""
    a = np.ascontiguousarray(action, np.float32)
    term = C.c_int()
    check(lib().dr_env_step(C.byref(env), true_theta, abi.fptr(a), C.byref(state), abi.fptr(belief), int(update_belief), seed, step, C.byref(term)),
          "dr_env_step")
    return term.value


def gate_env_step(env: abi.dr_gate_env_config, true_theta: int, action, state: abi.dr_gate_state, belief: np.ndarray, update_belief: bool, seed: int,
                  step: int):
    """One gate-race environment step on the device (dr_gate_env_step); returns
    (terminal type, new state, new belief)."""
    st = abi.dr_gate_state.from_buffer_copy(state)
    bel = np.zeros(abi.DR_MAX_THETA, np.float32)
    bel[: env.n_theta] = belief
    act = np.ascontiguousarray(action, np.float32)
    term = C.c_int()
    check(lib().dr_gate_env_step(C.byref(env), true_theta, abi.fptr(act), C.byref(st), abi.fptr(bel), int(update_belief), seed, step, C.byref(term)),
          "dr_gate_env_step")
    return term.value, st, bel[: env.n_theta].copy()
