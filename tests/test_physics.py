"""Physics checks in FP64 on the host (pyising_b200.physics), after src/pyising/validate.py.

CPU: the exact results are pinned to the reference's own values (tests/golden/exact.npz, made by
tests/golden/make_golden.py from src/pyising/exact.py) and the estimators to known cases.
GPU: a temperature scan and a Binder-cumulant scan run as batched ensembles and must agree with
the exact finite-torus energy, the Onsager-Yang magnetisation and the exact T_c.  The random
streams are fixed by the seeds, so every outcome is deterministic; the tolerances are several
standard errors (energy) or the known finite-size spread (magnetisation, crossing).
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import golden

from pyising_b200 import physics as ph


def test_exact_results_match_the_reference():
    """pyising takes the torus energy and specific heat as central differences of ln Z (steps
    1e-5 and 1e-4); the values here are analytic derivatives, so they agree within the
    truncation error of those differences (largest at L = 128 near T_c: ~6e-9 relative for
    the energy, ~5e-5 absolute for the specific heat)."""
    g = golden("exact.npz")
    for i, T in enumerate(g["T"]):
        for j, L in enumerate(g["L"]):
            assert ph.energy_torus(float(T), int(L)) == pytest.approx(g["energy_torus"][i, j],
                                                                       rel=2e-8)
            assert ph.specific_heat_torus(float(T), int(L)) == pytest.approx(
                g["specific_heat_torus"][i, j], rel=1e-4, abs=1e-6)
    np.testing.assert_allclose(ph.magnetization_2d(g["T"]), g["magnetization_2d"], rtol=1e-13)
    np.testing.assert_allclose(ph.energy_2d(g["T"]), g["energy_2d"], rtol=1e-13)


def _enumerated_torus(K: float, m: int, n: int) -> tuple[float, float, float]:
    """ln Z, <sum of bonds> and its variance of the m x n torus by summing all 2^(mn) states."""
    idx = np.arange(m * n).reshape(m, n)
    right, down = np.roll(idx, -1, axis=1).ravel(), np.roll(idx, -1, axis=0).ravel()
    states = ((np.arange(2 ** (m * n))[:, None] >> np.arange(m * n)) & 1) * 2 - 1
    bonds = (states * states[:, right]).sum(1) + (states * states[:, down]).sum(1)
    w = np.exp(K * (bonds - bonds.max()))
    z = w.sum()
    mean = float((w * bonds).sum() / z)
    var = float((w * bonds * bonds).sum() / z) - mean * mean
    return float(np.log(z)) + K * float(bonds.max()), mean, var


@pytest.mark.parametrize("m,n", [(4, 4), (4, 5), (3, 6)])
def test_kaufman_torus_equals_full_enumeration(m, n):
    """ln Z and its first two K-derivatives equal the sums over every state of small tori."""
    for K in (0.2, 0.35, ph.BETA_C_2D, 0.6, 1.0):
        lnz, mean, var = _enumerated_torus(K, m, n)
        assert ph.log_partition_torus(K, m, n) == pytest.approx(lnz, rel=1e-13)
        if m == n:
            assert ph.energy_torus(1.0 / K, m) == pytest.approx(-mean / (m * n), rel=1e-12)
            assert ph.specific_heat_torus(1.0 / K, m) == pytest.approx(K * K * var / (m * n),
                                                                        rel=1e-10)


def test_torus_energy_tends_to_onsager_away_from_tc():
    for T in (1.6, 2.0, 2.6, 3.5):
        assert ph.energy_torus(T, 128) == pytest.approx(float(ph.energy_2d(T)), abs=1e-6)
    assert ph.magnetization_2d(ph.TC_2D + 1e-9) == 0.0
    assert 0.0 < float(ph.magnetization_2d(ph.TC_2D - 1e-3)) < 0.6


def test_estimators_on_known_cases():
    rng = np.random.default_rng(5)
    assert ph.binder(np.array([1.0, -1.0] * 50)) == pytest.approx(2.0 / 3.0)
    assert abs(ph.binder(rng.normal(size=200000))) < 0.01  # Gaussian: U_4 = 0
    x = rng.normal(size=32 * 1000)
    assert ph.binning_error(x) == pytest.approx(1.0 / np.sqrt(x.size), rel=0.3)
    Ts = np.array([2.0, 2.1, 2.2, 2.3])
    # differences 0.05, 0.02, -0.01, -0.04: zero two thirds of the way from 2.1 to 2.2
    assert ph.crossing(Ts, [0.60, 0.62, 0.64, 0.66], [0.55, 0.60, 0.65, 0.70]) == pytest.approx(
        2.1 + 0.2 / 3)
    assert np.isnan(ph.crossing(Ts, [1, 1, 1, 1], [0, 0, 0, 0]))
    s = ph.Summary.from_series(np.array([[16, -32], [-16, -32], [16, -24], [16, -32]]), 16,
                               skip=0)
    assert s.abs_m == 1.0 and s.e == pytest.approx(-1.875)


@pytest.mark.gpu
def test_energy_scan_agrees_with_the_exact_torus():
    rows = ph.temperature_scan(128, [1.8, 2.6, 3.2], therm=2000, meas=4000, every=4)
    assert len(rows) == 9
    for r in rows:
        assert abs(r["e_z"]) < 4.5, r
        if r["T"] < ph.TC_2D:
            assert r["abs_m"] == pytest.approx(r["m_exact_inf"], abs=0.01), r


@pytest.mark.gpu
def test_binder_crossing_near_the_exact_tc():
    out = ph.binder_scan([8, 16], np.linspace(2.16, 2.38, 8), therm=4000, meas=20000, every=2)
    tx = out["crossings"]["8-16"]
    assert abs(tx - ph.TC_2D) < 0.05, out
    for L in (8, 16):
        u = out["U4"][L]
        assert u[0] > u[-1]  # ordered (U_4 -> 2/3) to disordered (U_4 -> 0)
        assert all(0.0 < x < 2.0 / 3.0 + 0.02 for x in u)
