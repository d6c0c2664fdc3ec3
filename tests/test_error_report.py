"""The error report's classification (thesiscode_b200/error_report.py) on small
synthetic cases: which windows count against the FP32 form and which are set
apart because the FP64 (reference) value is itself off."""
from __future__ import annotations

import numpy as np

from thesiscode_b200 import Profile, error_report, workloads


def _exact(oracle, x, m):
    d2, idx = oracle.selfjoin(x, m)
    return Profile(d2.copy(), idx.copy())


def test_identical_profiles_have_no_error(oracle):
    x = workloads.random_walk(2000, 3)
    m = 40
    p = _exact(oracle, x, m)
    rep = error_report.compare(x, m, [], p, Profile(p.dist2.copy(), p.index.copy()), False)
    assert rep["max_rel"] == 0.0 and rep["windows_over_tol"] == 0
    assert rep["index_agreement"] == 1.0


def test_fp32_error_is_counted(oracle):
    x = workloads.random_walk(2000, 4)
    m = 40
    p64 = _exact(oracle, x, m)
    p32 = Profile(p64.dist2.copy(), p64.index.copy())
    p32.dist2[100] *= (1 + 1e-3) ** 2  # distance off by 1e-3 relative
    rep = error_report.compare(x, m, [], p64, p32, False)
    assert rep["windows_over_tol"] == 1 and rep["reference_inaccurate"] == 0
    assert abs(rep["max_rel"] - 1e-3) < 1e-6


def test_inaccurate_reference_is_set_apart(oracle):
    x = workloads.random_walk(2000, 5)
    m = 40
    p32 = _exact(oracle, x, m)
    p64 = Profile(p32.dist2.copy(), p32.index.copy())
    p64.dist2[200] *= (1 + 1e-3) ** 2  # the FP64 value is off its own pair's distance
    rep = error_report.compare(x, m, [], p64, p32, False)
    assert rep["windows_over_tol"] == 1 and rep["reference_inaccurate"] == 1
    assert rep["max_rel"] < 1e-6 and rep["fp32_max_rel_vs_direct_on_those"] < 1e-6


def test_reference_missing_a_closer_neighbour_is_set_apart(oracle):
    x = workloads.random_walk(2000, 6)
    m = 40
    p32 = _exact(oracle, x, m)
    p64 = Profile(p32.dist2.copy(), p32.index.copy())
    w = 300
    # give the FP64 side a worse but self-consistent neighbour
    PL = x.size - m + 1
    cand = [j for j in range(PL) if abs(j - w) > m // 4 and j != p32.index[w]]
    d = np.array([error_report.pair_distance(x, m, w, j) for j in cand])
    k = int(np.argsort(d)[5])
    p64.index[w] = cand[k]
    p64.dist2[w] = d[k] ** 2
    rep = error_report.compare(x, m, [], p64, p32, False)
    assert rep["reference_inaccurate"] == 1 and rep["max_rel"] < 1e-6


def test_constant_stretches_are_reported_apart(oracle):
    x = workloads.random_walk(3000, 7)
    m = 32
    s = 1000
    x[s:s + 2 * m] = 0.0
    p = _exact(oracle, x, m)
    rep = error_report.compare(x, m, [(s, 2 * m)], p, Profile(p.dist2.copy(), p.index.copy()),
                               True)
    assert rep["flat_windows"] == m + 1
    assert rep["flat_convention_fp64"] and rep["flat_convention_fp32"]
    zone = error_report.stretch_zone(x.size - m + 1, m, [(s, 2 * m)], 100)
    assert zone[s - m - 100] and zone[s + 2 * m + 99] and not zone[s + 2 * m + 100]
