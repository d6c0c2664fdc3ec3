"""The PreSCRIMP restatement (oracle/prescrimp.py) on CPU.

- Against the reference itself: golden outputs of the reference's own
  ScrimpppOrig.cpp (tests/golden/prescrimp_ref.npz, made by
  tests/golden/make_prescrimp_golden.py with a stand-in FFT for FFTW) and, where
  oracle/_ref is built, a live run on a fresh series.  The reference forms each
  query row by FFT convolution, the restatement by direct dot products, so the
  distances agree to rounding (1e-9 relative) and a differing index must tie.
- With a step of one window every window is a query, so the profile is the
  exact brute-force profile under PreSCRIMP's exclusion rule (|i - j| < m/4
  excluded)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle.prescrimp import orig_stats, prescrimp
from thesiscode_b200 import workloads
from thesiscode_b200.error_report import pair_distance

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BINARY = os.path.join(ROOT, "oracle", "_ref", "scrimppp_ref_orig")


def check_against_reference(x, m, dist2, index, ref_dist, ref_index, rtol=1e-9):
    """(dist2, index) against the reference's (sqrt |d2|, index): same untouched
    windows (+inf, index 0), distances within rtol, and where the indices differ
    the two neighbours' distances agree within rtol."""
    d = np.sqrt(np.abs(dist2))
    fin = np.isfinite(ref_dist)
    assert np.array_equal(np.isfinite(d), fin)
    assert np.all(index[~fin] == 0) and np.all(ref_index[~fin] == 0)
    assert np.allclose(d[fin], ref_dist[fin], rtol=rtol, atol=0)
    for w in np.nonzero((index != ref_index) & fin)[0]:
        a = pair_distance(x, m, int(w), int(index[w]))
        b = pair_distance(x, m, int(w), int(ref_index[w]))
        assert a == pytest.approx(b, rel=rtol), (w, index[w], ref_index[w])


def golden_rtol(name: str) -> float:
    """Distance tolerance against the reference's FFT rows: 1e-9, except at a
    level offset of 1e4, where an FFT row's rounding (~1e-16 of |A| |query| ~
    1e9) divided by window variances of order 1 leaves ~2e-7 in the reference's
    own distances."""
    return 1e-6 if name.startswith("offset") else 1e-9


def test_restatement_matches_reference_golden(golden_prescrimp):
    assert len(golden_prescrimp) >= 8
    for name, c in golden_prescrimp.items():
        m, stride = int(c["m"]), int(c["stride"])
        d2, idx = prescrimp(c["x"], m, float(stride))
        check_against_reference(c["x"], m, d2, idx, c["dist"], c["index"].astype(np.int64),
                                rtol=golden_rtol(name))


@pytest.mark.skipif(not os.path.exists(REF_BINARY), reason="oracle/_ref not built (no reference tree)")
def test_restatement_matches_reference_live():
    from tests.golden.make_prescrimp_golden import run_reference
    for n, m, stride, seed in [(1800, 40, 1, 3), (1024, 24, 4, 4)]:
        x = workloads.random_walk(n, seed)
        ref_d, ref_i = run_reference(x, m, stride)
        d2, idx = prescrimp(x, m, float(stride))
        check_against_reference(x, m, d2, idx, ref_d, ref_i)


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
