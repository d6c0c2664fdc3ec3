"""The long drift/flat-stress workload (n = 8,388,608, m = 1024, 32 planted
sine motifs, 16 constant segments of 2m) at full length.

A whole CPU join of it takes hours, so parity with the reference is pinned on
diagonal ranges: the FP64 form over [lo, hi) equals the oracle's join over
the same diagonals with the reference's block geometry, bit for bit, at the
long-series index arithmetic (neighbour indices up to 8.4M, 24 index bits in
the packed keys).  Ranges cross a block boundary (blocklen 500), sit in the
middle, and end at the last diagonal."""
from __future__ import annotations

import numpy as np
import pytest

import thesiscode_b200 as mp
from thesiscode_b200 import error_report, workloads

from test_parity_gpu import check_fp64_indices

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c3():
    x, m, info = workloads.c3()
    return x, m, [(s, L) for kind, s, L in info if kind == "flat"]


@pytest.fixture(scope="module")
def c3z():
    x, m, info = workloads.c3(zero_level=True)
    return x, m, [(s, L) for kind, s, L in info if kind == "flat"]


def _ranges(PL, m):
    lo = m // 4 + 1
    # the first range crosses the block boundary at diagonal lo + 500
    return [(lo + 380, lo + 620), (PL // 2, PL // 2 + 150), (PL - 800, PL)]


def test_fp64_c3_diagonal_ranges_match_oracle(gpu_ctx, oracle, c3):
    x, m, _ = c3
    PL = x.size - m + 1
    for lo, hi in _ranges(PL, m):
        d2, idx = oracle.selfjoin(x, m, diag_lo=lo, diag_hi=hi)
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
        assert np.array_equal(p.dist2, d2), (lo, hi)
        check_fp64_indices(oracle, x, m, p.dist2, p.index, idx)


def test_fp64_c3_zero_level_flat_windows(gpu_ctx, oracle, c3z):
    x, m, segs = c3z
    PL = x.size - m + 1
    lo, hi = m // 4 + 1, m // 4 + 1 + 256
    d2, idx = oracle.selfjoin(x, m, diag_lo=lo, diag_hi=hi)
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
    assert np.array_equal(p.dist2, d2)
    check_fp64_indices(oracle, x, m, p.dist2, p.index, idx)
    flat = error_report.inside_constant(PL, m, segs)
    assert flat.sum() == 16 * (m + 1)
    assert np.all(p.dist2[flat] == 2.0 * m + 2.0) and np.all(p.index[flat] == 0)
    assert not np.any(flat[p.index[~flat]] & (p.dist2[~flat] < 2.0 * m + 2.0))


@pytest.mark.parametrize("K", [64, 1024])
def test_fp32_c3_ranges_within_tolerance(gpu_ctx, c3, c3z, K):
    """FP32 re-anchored vs FP64 on the same diagonals.  Away from the constant
    stretches (the window and both chosen neighbours farther than m + K from
    one), the distance error is <= 1e-4 relative wherever the FP64 value is
    itself accurate.  Windows inside a stretch give the flat result; at zero
    level both forms follow the reference's flat convention exactly."""
    for (x, m, segs), zero in ((c3, False), (c3z, True)):
        PL = x.size - m + 1
        for lo, hi in _ranges(PL, m):
            p64 = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
            p32 = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=K, diag_lo=lo,
                                   diag_hi=hi)
            rep = error_report.compare(x, m, segs, p64, p32, zero, K=K)
            assert rep["max_rel_far_from_stretches"] <= 1e-4, (zero, lo, hi, rep)
            assert rep["near_stretch_windows"] <= 0.02 * PL, rep
            if zero:
                assert rep["flat_convention_fp32"] and rep["flat_convention_fp64"], rep
                assert rep["no_window_points_at_flat_fp32"], rep
            else:
                assert rep["pseudo_flat_fp32_is_flat_result"], rep
