"""Bounded device waits: a staging wait that runs out is reported to the caller.

The rollout and verification CTAs stage the track and the plan in shared memory by bulk
copies that complete on an mbarrier, and wait for it a bounded number of polls. The test
switch dr_mppi_debug_stage_timeout makes every CTA announce its staging bytes without
issuing the copies (a flag that nothing sets: nothing is in flight), so the waits run out;
the step must then return DR_ERR_TIMEOUT with the count in info.verif_timeouts, and the
context must stay usable: with the switch off, the next step succeeds and equals the step
of an identical controller that never timed out.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import drb
from helpers import mppi_ctl, small_mppi

pytestmark = pytest.mark.gpu
abi = drb.abi


def _step(ctl, sc):
    out = np.zeros(2, np.float32)
    info = abi.dr_mppi_info()
    rc = abi.lib().dr_mppi_step(ctl.handle, C.byref(sc.state), abi.fptr(ctl.h_belief), abi.fptr(out), C.byref(info))
    return rc, out, info


@pytest.mark.parametrize("spl", [False, True])
def test_stage_timeout_is_reported_and_context_survives(gpu, spl):
    sc = small_mppi(spl, K=512, T=30, M=8, n_verif=1024)
    ctl = mppi_ctl(sc)
    twin = mppi_ctl(sc)
    ctl.engine = twin.engine = object()
    # step 1: both controllers step normally
    rc, a, _ = _step(ctl, sc)
    assert rc == abi.DR_OK
    rc, b, _ = _step(twin, sc)
    assert rc == abi.DR_OK and np.array_equal(a, b)
    # step 2 with the staging switch on: every rollout and verification CTA gives up
    abi.check(abi.lib().dr_mppi_debug_stage_timeout(ctl.handle, 1, 256), "stage_timeout on")
    rc, _, info = _step(ctl, sc)
    assert rc == abi.DR_ERR_TIMEOUT, abi.lib().dr_last_error()
    assert b"bounded device wait" in abi.lib().dr_last_error()
    assert info.verif_timeouts > 0
    # switch off: the context is usable and the controller steps again
    abi.check(abi.lib().dr_mppi_debug_stage_timeout(ctl.handle, 0, 0), "stage_timeout off")
    rc, a, info = _step(ctl, sc)
    assert rc == abi.DR_OK, abi.lib().dr_last_error()
    assert info.verif_timeouts == 0
    assert np.all(np.isfinite(a))


def test_timed_out_rollout_writes_defined_costs(gpu):
    """A timed-out rollout tile leaves infinite costs (never stale or uninitialised
    values) for the update to read."""
    sc = small_mppi(False, K=700, T=30, n_verif=512)
    ctl = mppi_ctl(sc)
    K, nth = sc.mppi.n_samples, sc.n_theta
    belief = sc.belief()
    costs = np.zeros((nth + 1, K), np.float32)
    abi.check(abi.lib().dr_mppi_debug_stage_timeout(ctl.handle, 1, 128), "stage_timeout on")
    abi.lib().dr_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), None, None, None, abi.fptr(costs))
    abi.check(abi.lib().dr_mppi_debug_stage_timeout(ctl.handle, 0, 0), "stage_timeout off")
    assert np.all(np.isinf(costs))
    abi.check(abi.lib().dr_mppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), None, None, None, abi.fptr(costs)), "rollout")
    assert np.all(np.isfinite(costs))
