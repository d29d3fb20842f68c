"""Edge cases of the MPPI path on the B200 against the CPU oracle port: the longest
horizon and the most knots accepted, sample and verification counts that fill no tile
evenly, a single sample, and the other compiled (n_opp, n_theta) combinations."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import O, drb
from helpers import OracleMPPI, mppi_ctl, random_nominal, small_mppi
from test_gpu_grad import _multi_scenario
from test_gpu_mppi import _dev_rollout

pytestmark = pytest.mark.gpu
abi = drb.abi


def _rollout_agreement(sc, ctl, spl):
    belief = sc.belief()
    kn = ctl.knots().copy()
    B = O.spline_matrix(sc.mppi) if spl else None
    noise = O.mppi_noise(sc, 0)
    ct, bu, bt, _ = _dev_rollout(ctl, sc, belief)
    oct32, obu, obt = O.mppi_rollout(sc, belief, kn, noise, B, 0, prec=32)
    rel = np.abs(ct - oct32) / np.maximum(1.0, np.abs(oct32))
    finite = np.isfinite(oct32)
    assert np.array_equal(np.isfinite(ct), finite)
    return float(np.mean(rel[finite] <= 1e-5)), float(np.mean(bu == obu))


@pytest.mark.parametrize("spl", [True, False])
def test_longest_horizon_most_knots_ragged_tiles(gpu, spl):
    """H = 256 (the largest accepted), 60 knots (the reference's MAX_N_KNOTS), K = 300
    and V = 777 (partial rollout and verification tiles)."""
    sc = small_mppi(spl, K=300, T=256, M=60, n_verif=777, noise=True)
    rng = np.random.default_rng(21)
    nominal = random_nominal(sc, rng, 0.3)
    ctl = mppi_ctl(sc, nominal=nominal)
    frac, bfrac = _rollout_agreement(sc, ctl, spl)
    print(f"spl={spl}: rollout agreement {frac:.4f}, branch bookkeeping {bfrac:.4f}")
    assert frac >= 0.97 and bfrac >= 0.97
    ctl2 = mppi_ctl(sc, nominal=nominal, exact_verify=True)
    ctl2.engine = object()
    ref = OracleMPPI(sc, nominal=nominal)
    a = ctl2.getControl(sc.state)
    oa, info = ref.get_control(sc.state, sc.belief())
    np.testing.assert_allclose(a, oa, rtol=2e-3, atol=2e-3)
    assert ctl2.useNewPlan == info["use_new"]


def test_single_sample_single_verification_sample(gpu):
    sc = small_mppi(False, K=1, T=40, n_verif=1, noise=True)
    ctl = mppi_ctl(sc)
    frac, _ = _rollout_agreement(sc, ctl, False)
    assert frac == 1.0
    ctl2 = mppi_ctl(sc, exact_verify=True)
    ctl2.engine = object()
    ref = OracleMPPI(sc)
    for _ in range(3):
        a = ctl2.getControl(sc.state)
        oa, info = ref.get_control(sc.state, sc.belief())
        np.testing.assert_allclose(a, oa, rtol=2e-3, atol=2e-3)
        assert ctl2.useNewPlan == info["use_new"]


@pytest.mark.parametrize("nopp,nth", [(2, 2), (1, 8), (1, 4), (1, 1)])
def test_other_sizes_ragged(gpu, nopp, nth):
    sc = _multi_scenario(nopp, nth, True)
    sc.mppi.n_samples = 129
    sc.seed = 3
    ctl = drb.controllers.MPPIController(sc.env, sc.mppi, sc.seed, nominal=random_nominal(sc, np.random.default_rng(nth), 0.3))
    frac, bfrac = _rollout_agreement(sc, ctl, True)
    print(f"nopp={nopp} nth={nth}: rollout agreement {frac:.4f}, branch bookkeeping {bfrac:.4f}")
    assert frac >= 0.97 and bfrac >= 0.97
