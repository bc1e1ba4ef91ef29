"""Blocking error of the mean against an AR(1) series with a known answer."""
import numpy as np
import pytest

from mpsqmc_b200 import analysis


def test_blocking_recovers_ar1_error_of_mean():
    rng = np.random.default_rng(5)
    phi, n, reps = 0.9, 1 << 14, 40
    # exact error of the mean of an AR(1) series with unit innovations, for large n:
    # sigma_x^2 (1 + phi) / (1 - phi) / n, sigma_x^2 = 1 / (1 - phi^2)
    exact = np.sqrt((1.0 / (1 - phi ** 2)) * (1 + phi) / (1 - phi) / n)
    est = []
    for _ in range(reps):
        x = np.empty(n)
        x[0] = rng.normal() / np.sqrt(1 - phi ** 2)
        eps = rng.normal(size=n)
        for t in range(1, n):
            x[t] = phi * x[t - 1] + eps[t]
        est.append(analysis.blocking_error(x))
    assert np.mean(est) == pytest.approx(exact, rel=0.15)


def test_uncorrelated_series_gives_naive_error():
    rng = np.random.default_rng(6)
    x = rng.normal(size=4096)
    assert analysis.blocking_error(x) == pytest.approx(1 / np.sqrt(4096), rel=0.25)


def test_variance_normalised_scales_with_throughput():
    rng = np.random.default_rng(7)
    e = -28.17 + 0.01 * rng.normal(size=500)
    a = analysis.variance_normalised(1000.0, e, np.full(500, 2048))
    b = analysis.variance_normalised(2000.0, e, np.full(500, 2048))
    assert b["vn"] == pytest.approx(2 * a["vn"])
    assert a["steps_used"] == 400 and a["equil_steps"] == 100


def test_proposal_gain_bound():
    from mpsqmc_b200 import analysis
    assert analysis.proposal_gain_bound([np.ones(10)]) == pytest.approx(1.0)
    w = np.array([1.0, 1.0, 2.0, 4.0])
    assert analysis.proposal_gain_bound([w, w]) == pytest.approx(4 * 22 / 64)
