"""The guarded FP32 form (MP_PREC_FP32_GUARDED): the FP32 re-anchored join plus
FP64 tiles around ill-conditioned windows, an FP64 pass over near-duplicates
and FP64 distances of the chosen pairs.

- on a plain random walk nothing is ill-conditioned: each neighbour is the
  best (by FP64) of the FP32 pass's winning group of adjacent candidates, so
  at least as many neighbours agree with the FP64 form's as in the plain FP32
  form, and every distance is the chosen pair's exact distance;
- on exact repeats (near-duplicates far below FP32 resolution) every window
  finds a partner at least as close as the FP64 form's, with exact distances;
- on the long stress series (constant stretches at the walk's level and at 0)
  the error against the FP64 form stays within 2e-4 on every window whose FP64
  value is itself accurate, near the stretches included."""
from __future__ import annotations

import numpy as np
import pytest

import thesiscode_b200 as mp
from thesiscode_b200 import error_report, workloads

from test_c3_gpu import _ranges

pytestmark = pytest.mark.gpu


def _direct(x, m, d2, idx, sample):
    got = np.sqrt(np.abs(d2[sample]))
    want = np.array([error_report.pair_distance(x, m, int(i), int(idx[i])) for i in sample])
    return got, want


def test_plain_walk_best_adjacent_neighbours_exact_distances(gpu_ctx):
    x = workloads.random_walk(200_000, 21)
    m = 128
    p64 = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    p32 = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=1024)
    pg = gpu_ctx.selfjoin(x, m, precision=mp.FP32_GUARDED, reanchor_k=1024)
    assert gpu_ctx.last_near_duplicates == 0
    assert np.mean(pg.index == p64.index) >= np.mean(p32.index == p64.index)
    d64 = np.sqrt(p64.dist2)
    assert np.max(np.abs(np.sqrt(pg.dist2) - d64) / d64) <= 1e-4
    sample = np.random.default_rng(0).choice(x.size - m + 1, 2000, replace=False)
    got, want = _direct(x, m, pg.dist2, pg.index, sample)
    assert np.allclose(got, want, rtol=1e-9, atol=1e-12)


def test_exact_repeats_are_resolved(gpu_ctx):
    rng = np.random.default_rng(8)
    base = np.cumsum(rng.standard_normal(1500))
    x = np.concatenate([base + 3.0 * k + rng.normal(0, 1e-3, base.size) for k in range(4)])
    m = 100
    p64 = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    pg = gpu_ctx.selfjoin(x, m, precision=mp.FP32_GUARDED, reanchor_k=256)
    assert gpu_ctx.last_near_duplicates > 0
    sample = np.arange(0, x.size - m + 1, 7)
    got, want = _direct(x, m, pg.dist2, pg.index, sample)
    assert np.allclose(got, want, rtol=1e-4)
    # the plain FP32 form cannot rank these (u ~ 1e-7, its resolution floor)
    p32 = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=256)
    g32, w32 = _direct(x, m, p32.dist2, p32.index, sample)
    assert np.max(np.abs(g32 - w32) / w32) > 1e-2
    ref, _ = _direct(x, m, p64.dist2, p64.index, sample)
    assert np.all(want <= ref * (1 + 1e-4))  # never a worse partner than the FP64 form


@pytest.mark.parametrize("K", [256, 1024])
def test_stress_series_within_tolerance(gpu_ctx, K):
    from test_c3_gpu import workloads as wl
    for zero in (False, True):
        x, m, info = wl.c3(zero_level=zero)
        segs = [(s, L) for kind, s, L in info if kind == "flat"]
        PL = x.size - m + 1
        for lo, hi in _ranges(PL, m):
            p64 = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
            pg = gpu_ctx.selfjoin(x, m, precision=mp.FP32_GUARDED, reanchor_k=K, diag_lo=lo,
                                  diag_hi=hi)
            rep = error_report.compare(x, m, segs, p64, pg, zero, K=K)
            assert rep["max_rel"] <= 2e-4, (zero, lo, hi, rep)
            if zero:
                assert rep["flat_convention_fp32"], rep
            else:
                assert rep["pseudo_flat_fp32_is_flat_result"], rep


def test_default_interval_meets_bound_far_from_stretches(gpu_ctx):
    """At its default re-anchor interval (reanchor_k = 0 -> 512) the guarded
    form's distances stay within 1e-4 of the FP64 form's away from the
    constant stretches, on both stress series and every sampled range; near
    them as well."""
    for zero in (False, True):
        x, m, info = workloads.c3(zero_level=zero)
        segs = [(s, L) for kind, s, L in info if kind == "flat"]
        PL = x.size - m + 1
        for lo, hi in _ranges(PL, m):
            p64 = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
            pg = gpu_ctx.selfjoin(x, m, precision=mp.FP32_GUARDED, diag_lo=lo, diag_hi=hi)
            rep = error_report.compare(x, m, segs, p64, pg, zero, K=512)
            assert rep["max_rel_far_from_stretches"] <= 1e-4, (zero, lo, hi, rep)
            assert rep["max_rel_near_stretches"] <= 1e-4, (zero, lo, hi, rep)
