"""Gradient path of the MPPI controller, as a torch op.

The objective is the one `dr_mppi_nominal_grad` (include/drmppi.h) evaluates on the
device: the belief-weighted cost of the noise-free rollout of a control sequence U
((n_theta+1) x M x 2 spline knots, or dense controls) from a state, rolled out and costed
as the reference's fullRolloutKernel does (src/kernels.cu:34-171, include/costs.cuh:7-39).
Its gradient with respect to U and to the six cost weights comes from the library's
adjoint kernel (a reverse sweep over the horizon with state checkpoints).

    J = nominal_cost(ctl, state, belief, U, w)          # differentiable in U and w

`U` has shape (n, n_theta+1, M, 2) or (n_theta+1, M, 2); `w` (n, 6) or (6,) in the order
of WEIGHT_NAMES (None: the controller's own weights, not differentiated). Tensors live on
the controller's CUDA device; the op runs on torch's current stream.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi
from .abi import check, lib

WEIGHT_NAMES = ("boundary_cost", "outside_cost", "win_cost", "opp_win_cost", "final_adv_weight", "final_opp_adv_weight")


def weights_of(cfg: abi.dr_mppi_config) -> list[float]:
    """The six differentiable cost weights of an MPPI configuration, in WEIGHT_NAMES order."""
    return [float(getattr(cfg, n)) for n in WEIGHT_NAMES]


def _state_bytes(state) -> torch.Tensor:
    if not isinstance(state, abi.dr_sim_state):
        raise TypeError("the gradient path takes a dr_sim_state (strategic race)")
    return torch.frombuffer(bytearray(bytes(state)), dtype=torch.uint8)


@torch.library.custom_op("drone_race_b200::nominal_cost_grad", mutates_args=(), device_types="cuda")
def nominal_cost_grad(handle: int, state: torch.Tensor, belief: torch.Tensor, knots: torch.Tensor, weights: torch.Tensor, use_weights: bool,
                      ckpt: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """(J [n], dJ/dU [n, nbp, M, 2], dJ/dw [n, 6]) for n start points `knots` (CUDA,
    float32, contiguous). `state`: the dr_sim_state bytes (CPU uint8); `belief`: CPU
    float32; `weights` [n, 6] CUDA float32, used when `use_weights`."""
    if knots.dtype != torch.float32 or not knots.is_cuda or knots.dim() != 4:
        raise ValueError("knots: a CUDA float32 tensor of shape (n, n_theta+1, M, 2)")
    knots = knots.contiguous()
    n = knots.shape[0]
    st = abi.dr_sim_state.from_buffer_copy(bytes(state.cpu().numpy().tobytes()))
    bel = belief.detach().cpu().to(torch.float32).contiguous().numpy()
    J = torch.empty(n, dtype=torch.float32, device=knots.device)
    dU = torch.empty_like(knots)
    dW = torch.empty((n, abi.DR_GRAD_WEIGHTS), dtype=torch.float32, device=knots.device)
    w = weights.contiguous() if use_weights else None
    stream = torch.cuda.current_stream(knots.device).cuda_stream
    check(lib().dr_mppi_nominal_grad(C.c_void_p(handle), C.byref(st), abi.fptr(bel), n, C.c_void_p(knots.data_ptr()),
                                     C.c_void_p(w.data_ptr()) if w is not None else None, C.c_void_p(J.data_ptr()), C.c_void_p(dU.data_ptr()),
                                     C.c_void_p(dW.data_ptr()), ckpt, C.c_void_p(stream)), "dr_mppi_nominal_grad")
    return J, dU, dW


@nominal_cost_grad.register_fake
def _(handle, state, belief, knots, weights, use_weights, ckpt):
    n = knots.shape[0]
    return (knots.new_empty(n), torch.empty_like(knots), knots.new_empty((n, abi.DR_GRAD_WEIGHTS)))


class NominalCost(torch.autograd.Function):
    """J(U, w) with the adjoint kernel's gradients as the backward pass."""

    @staticmethod
    def forward(ctx, handle, state, belief, knots, weights, use_weights, ckpt):
        J, dU, dW = nominal_cost_grad(handle, state, belief, knots, weights, use_weights, ckpt)
        ctx.save_for_backward(dU, dW)
        ctx.use_weights = use_weights
        return J

    @staticmethod
    def backward(ctx, gJ):
        dU, dW = ctx.saved_tensors
        gU = gJ.reshape(-1, 1, 1, 1) * dU
        gW = gJ.reshape(-1, 1) * dW if ctx.use_weights else None
        return None, None, None, gU, gW, None, None


def nominal_cost(ctl, state, belief, knots: torch.Tensor, weights: torch.Tensor | None = None, ckpt: int = 0) -> torch.Tensor:
    """Differentiable objective of controller `ctl` (an MPPIController on the strategic
    race) at the control sequences `knots` and cost weights `weights`."""
    single = knots.dim() == 3
    U = knots.unsqueeze(0) if single else knots
    use_w = weights is not None
    if use_w:
        W = weights.unsqueeze(0) if weights.dim() == 1 else weights
        W = W.expand(U.shape[0], abi.DR_GRAD_WEIGHTS)
    else:
        W = U.new_zeros((U.shape[0], abi.DR_GRAD_WEIGHTS))
    bel = torch.as_tensor(belief, dtype=torch.float32).reshape(-1)
    J = NominalCost.apply(int(ctl.handle.value), _state_bytes(state), bel, U, W, use_w, int(ckpt))
    return J[0] if single else J
