"""The PreSCRIMP restatement (oracle/prescrimp.py) on CPU: with a step of one
window every window is a query, so its profile is the exact brute-force
profile under PreSCRIMP's exclusion rule (|i - j| < m/4 excluded)."""
from __future__ import annotations

import numpy as np

from oracle.prescrimp import orig_stats, prescrimp
from thesiscode_b200 import workloads


def _brute(x, m):
    n = x.size
    PL = n - m + 1
    W = np.lib.stride_tricks.sliding_window_view(x, m)
    Z = (W - W.mean(axis=1, keepdims=True)) / W.std(axis=1, keepdims=True)
    D = 2.0 * m * (1.0 - (Z @ Z.T) / m)
    excl = m // 4
    ii, jj = np.meshgrid(np.arange(PL), np.arange(PL), indexing="ij")
    D[np.abs(ii - jj) < excl] = np.inf
    return D.min(axis=1), D.argmin(axis=1)


def test_every_window_a_query_gives_the_exact_profile():
    x = workloads.random_walk(900, 5)
    m = 32
    d2, idx = prescrimp(x, m, 1.0 / m)  # step floor(stride * m) = 1
    bd, bi = _brute(x, m)
    assert np.allclose(np.sqrt(np.abs(d2)), np.sqrt(np.abs(bd)), rtol=1e-8, atol=1e-9)
    assert np.mean(idx == bi) > 0.99


def test_sparser_queries_only_upper_bound_the_profile():
    x = workloads.random_walk(1500, 6)
    m = 40
    bd, _ = _brute(x, m)
    for stride in (0.25, 1.0, 5.0):
        d2, idx = prescrimp(x, m, stride)
        fin = np.isfinite(d2)
        assert fin.all()  # every window lies in some query's row
        assert np.all(d2 >= bd - 1e-8 * np.abs(bd) - 1e-9)


def test_orig_stats_are_prefix_sum_differences():
    x = workloads.random_walk(500, 7)
    mean, sigma = orig_stats(x, 20)
    W = np.lib.stride_tricks.sliding_window_view(x, 20)
    assert np.allclose(mean, W.mean(axis=1), rtol=1e-12)
    assert np.allclose(sigma, W.std(axis=1), rtol=1e-6)
