"""Autocorrelation analysis on series with known integrated times (no GPU)."""
import numpy as np

from pygcmc_b200 import analysis as A
from pygcmc_b200.values import StepLog_dtype


def ar1(phi, n, seed):
    g = np.random.default_rng(seed)
    x = np.empty(n)
    x[0] = g.normal()
    e = g.normal(size=n) * np.sqrt(1 - phi * phi)
    for t in range(1, n):
        x[t] = phi * x[t - 1] + e[t]
    return x


def test_integrated_time_of_ar1():
    # AR(1) with coefficient phi: tau = (1 + phi) / (1 - phi)
    for phi in (0.0, 0.5, 0.9):
        tau = A.integrated_time(ar1(phi, 200_000, 1))
        exact = (1 + phi) / (1 - phi)
        assert abs(tau - exact) / exact < 0.1, (phi, tau, exact)


def test_count_series_follows_logs():
    logs = np.zeros(4, dtype=StepLog_dtype)
    logs["ftype"] = [0, 1, 0, 1]
    logs["n_after"] = [3, 5, 2, 6]
    assert list(A.count_series(logs, [1, 4])) == [7, 8, 7, 8]
