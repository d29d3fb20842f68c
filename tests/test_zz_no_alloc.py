"""The allocation-free rollout entry point (dr_mppi_rollout_costs_noalloc), for callers
that cannot call cudaMalloc: through the C ABI, two calls in a row must give exactly the
per-branch sample costs of the regular entry point (dr_mppi_debug_rollout) on the same
controls, state, belief and random stream. Collected last on purpose (file name)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import drb
from helpers import mppi_ctl, random_nominal, small_mppi

pytestmark = pytest.mark.gpu
abi = drb.abi


def _regular_costs(ctl, sc, belief):
    K, nth = sc.mppi.n_samples, sc.n_theta
    costs = np.zeros((nth + 1, K), np.float32)
    abi.check(abi.lib().dr_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), None, None, None, abi.fptr(costs)), "debug_rollout")
    return costs


@pytest.mark.parametrize("spl,confident", [(False, False), (True, False), (False, True)])
def test_noalloc_rollout_matches_regular_entry_point(gpu, spl, confident):
    """confident: a belief above the confidence threshold commits every sample to the
    second hypothesis's branch, so the first branch has no compatible sample and its costs
    are infinite: the non-finite costs reach the caller as the regular path reports them."""
    import torch

    sc = small_mppi(spl, K=1500, T=40, M=10, noise=True)
    rng = np.random.default_rng(21)
    ctl = mppi_ctl(sc, nominal=random_nominal(sc, rng))
    belief = np.array([0.02, 0.98] if confident else [0.35, 0.65], np.float32)
    expect = _regular_costs(ctl, sc, belief)
    if confident:
        assert np.isinf(expect[1]).all()
    knots = torch.from_numpy(np.ascontiguousarray(ctl.knots())).cuda()
    for _ in range(2):
        out = torch.full((sc.n_theta + 1, sc.mppi.n_samples), float("nan"), dtype=torch.float32, device="cuda")
        rc = abi.lib().dr_mppi_rollout_costs_noalloc(C.byref(sc.env), C.byref(sc.mppi), sc.seed, 0, C.byref(sc.state), abi.fptr(belief),
                                                     C.c_void_p(knots.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert rc == abi.DR_OK, abi.lib().dr_last_error()
        got = out.cpu().numpy()
        same = (got == expect) | (np.isnan(got) & np.isnan(expect))
        assert same.all(), f"{(~same).sum()} of {got.size} costs differ"


def test_noalloc_rejects_problems_beyond_the_static_scratch(gpu):
    import torch

    sc = small_mppi(False, K=600_000, T=40, noise=True)
    knots = torch.zeros((sc.n_theta + 1, 40, 2), dtype=torch.float32, device="cuda")
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = abi.lib().dr_mppi_rollout_costs_noalloc(C.byref(sc.env), C.byref(sc.mppi), sc.seed, 0, C.byref(sc.state), abi.fptr(sc.belief()),
                                                 C.c_void_p(knots.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == abi.DR_ERR_INVALID_ARG
    assert b"static scratch" in abi.lib().dr_last_error()
