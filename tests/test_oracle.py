"""The oracle, pinned: the CPU restatement (oracle/port) reproduces, bit for bit, outputs
that the reference's own code produced (golden fixtures made by tests/golden/gen_golden.py
from the reference's model functions and its Python front-end), and its random streams
match the published Philox known-answer vectors."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from conftest import O, drb
from helpers import small_mppi

GOLD = Path(__file__).resolve().parent / "golden"
abi = drb.abi
S = drb.scenarios


def test_philox_known_answers():
    """Random123 kat_vectors for philox4x32_10."""
    out = (C.c_uint32 * 4)()
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0), (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, expect in cases:
        O.port().orc_philox(*ctr, *key, out)
        assert tuple(out) == expect


def test_normal_variates_are_standard_normal():
    from scipy import stats

    rng = np.random.default_rng(0)
    words = rng.integers(0, 2**32, size=400_000, dtype=np.uint64).astype(np.uint32)
    z = np.zeros(words.size, np.float32)
    O.port().orc_normals_from_words(O._u(words), words.size, O._f(z))
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
    assert stats.kstest(z, "norm").pvalue > 1e-3
    # inverse-CDF accuracy against scipy: the rational approximation evaluated in float
    # is accurate to ~1e-4 (plenty for sampling; both sides evaluate the same float ops)
    u = ((2 * (words[:20000] >> 9).astype(np.float64) + 1) * 2.0**-24)
    np.testing.assert_allclose(z[:20000], stats.norm.ppf(u), atol=3e-4, rtol=3e-4)


def test_series_log():
    x = np.exp(np.random.default_rng(1).uniform(np.log(6e-8), 0, 5000)).astype(np.float32)
    y = np.array([O.port().orc_series_logf(float(v)) for v in x], np.float64)
    np.testing.assert_allclose(y, np.log(x.astype(np.float64)), rtol=4e-7, atol=1e-7)


def test_track_grids_match_reference_front_end():
    """python-src/utils.py:391-427 on the reference's round track."""
    g = np.load(GOLD / "tracks.npz")
    mine = drb.track.track_grids(drb.track.circle_track(6.0))
    assert mine.track_length == pytest.approx(float(g["track_length"]), rel=1e-7)
    for name in ("p_grid", "dp_grid", "t_grid", "kappa_grid"):
        np.testing.assert_array_equal(getattr(mine, name), g[name].astype(np.float32))


@pytest.mark.parametrize("variant,spl", [("nth2_spline", True), ("nth2_dense", False)])
def test_mppi_oracle_matches_reference_golden(variant, spl):
    g = np.load(GOLD / f"mppi_{variant}.npz")
    sc = small_mppi(spl, K=64, T=24, M=8, n_verif=256, seed=int(g["seed"]), noise=True)
    step = int(g["step"])
    noise = O.mppi_noise(sc, step)
    assert np.array_equal(noise, g["noise"])
    B = O.spline_matrix(sc.mppi) if spl else None
    if spl:
        assert np.array_equal(B, g["B"])
    ct, bu, bt = O.mppi_rollout(sc, g["belief"], g["knots_in"], noise, B, step, prec=32)
    assert np.array_equal(ct, g["costs_true"])
    assert np.array_equal(bu, g["branch_used"]) and np.array_equal(bt, g["branch_time"])
    kn, dense, mins, nu, costs = O.mppi_update(sc, g["belief"], ct, bu, bt, noise, B, g["knots_in"], prec=32)
    assert np.array_equal(kn.astype(np.float32), g["knots_out"])
    assert np.array_equal(dense.astype(np.float32), g["dense"])
    assert np.array_equal(mins.astype(np.float32), g["min_costs"])
    assert np.array_equal(nu.astype(np.float32), g["nu"])
    assert np.array_equal(costs.astype(np.float32), g["costs"])
    fc, ft, _ = O.mppi_verify(sc, g["belief"], g["plan"].astype(np.float64), step, 1, prec=32)
    assert np.array_equal(fc, g["fail_count"]) and np.array_equal(ft, g["fail_time"])


@pytest.mark.parametrize("variant,nth", [("nth2_spline", 2), ("nth8_spline", 8)])
def test_prmppi_oracle_matches_reference_golden(variant, nth):
    g = np.load(GOLD / f"pr_{variant}.npz")
    if nth == 2:
        sc = S.strat_race(use_pr=True, K=64, T=24)
        sc.prmppi = S.make_prmppi(K=64, T=24, P=8, inv_temperature=1.0, sampling_noise=1.0)
    else:
        sc = S.robust_race(agent=1, seed=2, K=64, T=24, P=8, n_theta=nth)
    step = int(g["step"])
    assert np.array_equal(O.pr_noise(sc, step), g["noise"])
    assert np.array_equal(O.pr_thetas(sc, step, g["belief"]), g["thetas"])
    cn, cr = O.pr_rollout(sc, g["nom"], g["rob"], g["noise"], g["thetas"], step, prec=32)
    assert np.array_equal(cn, g["cost_nom"]) and np.array_equal(cr, g["cost_rob"])
    full, safe = O.pr_candidates(sc, g["nom"], g["rob"], g["thetas"], step, O.S_PR_CAND_ENV, prec=32)
    assert np.array_equal(full, g["cand_full"]) and np.array_equal(safe, g["cand_safe"])


def test_fp32_against_fp64_transcription():
    """FP32 error against the FP64 transcription of the same rollout, stated per output."""
    g = np.load(GOLD / "mppi_nth2_dense.npz")
    sc = small_mppi(False, K=64, T=24, M=8, n_verif=256, seed=int(g["seed"]), noise=True)
    ct32, _, _ = O.mppi_rollout(sc, g["belief"], g["knots_in"], g["noise"], None, int(g["step"]), prec=32)
    ct64, _, _ = O.mppi_rollout(sc, g["belief"], g["knots_in"], g["noise"], None, int(g["step"]), prec=64)
    rel = np.abs(ct32 - ct64) / np.maximum(1.0, np.abs(ct64))
    print(f"rollout cost FP32 vs FP64: median rel {np.median(rel):.2e}, 99th pct {np.percentile(rel, 99):.2e}")
    assert np.median(rel) < 1e-5


def test_clopper_pearson_bounds_against_scipy():
    g = np.load(GOLD / "cp.npz")
    for k, n, a, lo, hi in zip(g["k"], g["n"], g["alpha"], g["lower"], g["upper"]):
        assert O.port().orc_cp_lower(int(k), int(n), float(a)) == pytest.approx(lo, rel=1e-9, abs=1e-14)
        assert O.port().orc_cp_upper(int(k), int(n), float(a)) == pytest.approx(hi, rel=1e-9, abs=1e-14)


@pytest.mark.skipif(not O.ref_available("nth2_spline"), reason="reference build not present")
@pytest.mark.parametrize("spl", [True, False])
def test_oracle_port_equals_reference_host_code_live(spl):
    """Larger random case, port vs the reference's model functions compiled here."""
    variant = O.ref_variant_name(2, spl)
    sc = small_mppi(spl, K=256, T=40, n_verif=512, seed=99, noise=True)
    rng = np.random.default_rng(7)
    M = O.mk(sc.mppi)
    knots = rng.normal(0, 1.0, (3, M, 2)).astype(np.float32)
    noise = O.mppi_noise(sc, 5)
    B = O.spline_matrix(sc.mppi) if spl else None
    a = O.mppi_rollout(sc, np.array([0.6, 0.4], np.float32), knots, noise, B, 5, prec=32)
    b = O.mppi_rollout(sc, np.array([0.6, 0.4], np.float32), knots, noise, B, 5, impl=variant, nthreads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
