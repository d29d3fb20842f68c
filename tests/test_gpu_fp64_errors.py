"""FP32 (the CUDA path) against FP64 (the oracle's transcription of the same model, same
injected perturbations), stated per output: per-sample rollout costs, the updated control
sequence, the argmin sample of each branch plan outside near-ties, and PR-MPPI's running
and safety costs. The printed figures are the ones the design notes quote; the asserts
bound them."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import O, drb
from helpers import mppi_ctl, random_nominal, small_mppi
from test_gpu_mppi import _dev_noise, _dev_rollout
from test_gpu_prmppi import _noise_thetas, small_pr

pytestmark = pytest.mark.gpu
abi = drb.abi


def _rel(a, b):
    return np.abs(a - b) / np.maximum(1.0, np.abs(b))


@pytest.mark.parametrize("spl", [True, False])
def test_mppi_fp32_vs_fp64_per_output(gpu, spl):
    sc = small_mppi(spl, K=2048, T=40, noise=False)
    rng = np.random.default_rng(31)
    ctl = mppi_ctl(sc, nominal=random_nominal(sc, rng, 0.5))
    belief = np.array([0.4, 0.6], np.float32)
    B = O.spline_matrix(sc.mppi) if spl else None
    noise = _dev_noise(ctl, sc)
    # per-sample costs
    ct, bu, bt, costs = _dev_rollout(ctl, sc, belief)
    kn = ctl.knots().copy()  # the knots the rollout used
    ct64, bu64, bt64 = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=64)
    same = (bu == bu64) & (bt == bt64) & np.isfinite(ct) & np.isfinite(ct64)
    r = _rel(ct.astype(np.float64), ct64)[same]
    # updated control sequence: the GPU update on the GPU costs against the FP64 update
    # on the FP64 costs
    nbp, T, M = sc.n_theta + 1, sc.mppi.n_timesteps, O.mk(sc.mppi)
    dense = np.zeros((nbp, T, 2), np.float32)
    mins = np.zeros((nbp, M), np.float32)
    nu = np.zeros(nbp, np.float32)
    abi.check(abi.lib().dr_mppi_debug_update(ctl.handle, abi.fptr(belief), abi.fptr(np.ascontiguousarray(ct)), abi.iptr(bu), abi.iptr(bt),
                                             abi.fptr(dense), abi.fptr(mins), abi.fptr(nu)), "debug_update")
    new_kn = ctl.knots()
    kn64, dense64, mins64, nu64, costs64 = O.mppi_update(sc, belief, ct64, bu64, bt64, noise, B, kn, prec=64)
    scale = max(1e-6, float(np.abs(kn64 - kn).max()))  # size of the update itself
    du = float(np.abs(new_kn - kn64).max())
    dd = float(np.abs(dense - dense64).max())
    rnu = float(np.max(_rel(nu.astype(np.float64), nu64)))
    # argmin sample per branch plan, outside near-ties (FP64 gap between the two best
    # samples above 1e-5 relative)
    agree = ties = 0
    for b in range(nbp):
        c64 = costs64[b]
        fin = np.isfinite(c64)
        if fin.sum() < 2:
            continue
        order = np.argsort(np.where(fin, c64, np.inf))
        gap = (c64[order[1]] - c64[order[0]]) / max(1.0, abs(c64[order[0]]))
        if gap <= 1e-5:
            ties += 1
            continue
        agree += int(np.argmin(np.where(np.isfinite(costs[b]), costs[b], np.inf)) == order[0])
        assert np.argmin(np.where(np.isfinite(costs[b]), costs[b], np.inf)) == order[0], b
    print(f"spl={spl}: per-sample cost |fp32-fp64|/max(1,|fp64|): median {np.median(r):.2e} p99 {np.quantile(r, 0.99):.2e} max {r.max():.2e} "
          f"({same.mean():.4f} of samples with equal branch records); updated controls max |fp32-fp64| {du:.2e} "
          f"(update size {scale:.3g}); dense plan {dd:.2e}; nu rel {rnu:.2e}; argmin equal on {agree} branch plans, {ties} near-ties")
    assert same.mean() >= 0.97
    assert np.median(r) < 1e-5 and np.quantile(r, 0.99) < 1e-3
    # the weights exp(-(c - min) / lambda) turn the costs' FP32 rounding into a weight
    # error of |dc| / lambda, so the update's FP32-FP64 gap is bounded loosely
    assert du <= 0.05 * max(1.0, float(np.abs(kn64).max()))
    assert rnu < 0.05


def test_pr_fp32_vs_fp64_per_output(gpu):
    sc = small_pr(8, K=2048, T=64, noise=False)
    rng = np.random.default_rng(32)
    nominal = rng.normal(0, 0.8, (sc.prmppi.n_timesteps, 2)).astype(np.float32)
    ctl = drb.controllers.PRMPPIController(sc.env, sc.prmppi, sc.seed, nominal=nominal)
    belief = sc.belief()
    noise, th = _noise_thetas(ctl, sc, belief)
    c = sc.prmppi
    cn = np.zeros((c.P, c.n_samples, 2), np.float32)
    cr = np.zeros_like(cn)
    abi.check(abi.lib().dr_prmppi_debug_rollout(ctl.handle, C.byref(sc.state), abi.fptr(belief), abi.fptr(cn), abi.fptr(cr)), "pr debug_rollout")
    shifted = np.concatenate([nominal[1:], np.zeros((1, 2), np.float32)])
    cn64, cr64 = O.pr_rollout(sc, shifted, shifted, noise, th, 9, prec=64)
    out = []
    for name, a, b in (("nominal", cn, cn64), ("robust", cr, cr64)):
        for k, what in ((0, "running"), (1, "safety")):
            x, y = a[..., k].astype(np.float64), b[..., k]
            fin = np.isfinite(x) & np.isfinite(y)
            r = _rel(x, y)[fin]
            out.append(f"{name} {what}: median {np.median(r):.2e} p99 {np.quantile(r, 0.99):.2e} max {r.max():.2e}")
            assert np.median(r) < 1e-5 and np.quantile(r, 0.99) < 1e-3
    print("PR-MPPI |fp32-fp64|/max(1,|fp64|): " + "; ".join(out))
