"""The CPU oracle (oracle/scrimp_oracle.c) pinned against the reference's own
outputs: golden vectors recorded from the reference binaries, and -- where the
reference tree is built in this container -- the reference functions called
side by side."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle.oracle import RefOracle
from thesiscode_b200 import workloads


@pytest.mark.parametrize("m", [16, 64, 400])
def test_selfjoin_matches_reference_golden(oracle, golden_ascii, m):
    x = golden_ascii["series"]
    d2, idx = oracle.selfjoin(x, m)
    assert np.array_equal(d2, golden_ascii[f"d2_m{m}"])  # bit-identical values
    assert np.array_equal(idx, golden_ascii[f"idx_m{m}"])


def test_window_stats_and_first_qt_match_golden(oracle, golden_ascii):
    x = golden_ascii["series"]
    muS, sInv = oracle.window_stats(x, 64)
    assert np.array_equal(muS, golden_ascii["muS_m64"])
    assert np.array_equal(sInv, golden_ascii["sInv_m64"])
    qt = oracle.first_qt(x, 64, 0, 2000)
    assert np.array_equal(qt, golden_ascii["qt_m64_0_2000"])


def test_fast_math_reference_build_within_tolerance(golden_ascii):
    # the reference's release build (fast-math) differs from its IEEE build by
    # rounding noise only; recorded when the goldens were made
    for m in (16, 64, 400):
        assert float(golden_ascii[f"fast_maxrel_m{m}"]) < 1e-10
        assert int(golden_ascii[f"fast_idxdiff_m{m}"]) == 0


def test_edge_cases_match_reference(oracle, golden_edges):
    for name, c in golden_edges.items():
        m, B = (int(v) for v in c["meta"])
        d2, idx = oracle.selfjoin(c["x"], m, blocklen=B)
        ref = c["d2"]
        assert d2.shape == ref.shape, name
        assert np.array_equal(d2, ref, equal_nan=True), name
        # indices: identical unless the reference's shuffled block order broke
        # an exact tie differently
        diff = np.nonzero(idx != c["idx"])[0]
        for i in diff:
            a = oracle.pair_d2(c["x"], m, i, idx[i])
            b = oracle.pair_d2(c["x"], m, i, c["idx"][i])
            assert a == pytest.approx(b, rel=1e-9, abs=1e-12), (name, i)


def test_flat_zero_level_convention(oracle, golden_edges):
    c = golden_edges["flat_zero_level"]
    m = int(c["meta"][0])
    d2, idx = oracle.selfjoin(c["x"], m)
    x = c["x"]
    flat = np.array([np.all(x[i:i + m] == x[i]) for i in range(x.size - m + 1)])
    assert flat.any()
    # a zero-variance window keeps score -1 (d2 = 2m+2) and index 0 ...
    assert np.all(d2[flat] == 2 * m + 2)
    assert np.all(idx[flat] == 0)
    # ... and is never chosen as a neighbour
    assert not np.any(flat[idx[~flat]])


def test_n_equals_m_and_single_diagonal(oracle, golden_edges):
    c = golden_edges["n_equals_m"]
    d2, idx = oracle.selfjoin(c["x"], int(c["meta"][0]))
    assert d2.shape == (1,) and d2[0] == 2 * int(c["meta"][0]) + 2 and idx[0] == 0
    c = golden_edges["single_diagonal"]
    m = int(c["meta"][0])
    d2, idx = oracle.selfjoin(c["x"], m)
    assert np.array_equal(d2, c["d2"])


def test_c1_digest(oracle, digests):
    x, m = workloads.c1()
    d2, idx = oracle.selfjoin(x, m)
    assert hashlib.sha256(d2.tobytes()).hexdigest() == digests["c1"]["d2_sha256"]
    assert hashlib.sha256(idx.tobytes()).hexdigest() == digests["c1"]["idx_sha256"]


def test_restricted_range_equals_full_join_on_its_cells(oracle):
    x = workloads.random_walk(3000, 7)
    m = 40
    full, _ = oracle.selfjoin(x, m)
    a, _ = oracle.selfjoin(x, m, diag_lo=11, diag_hi=900)
    b, _ = oracle.selfjoin(x, m, diag_lo=900, diag_hi=x.size - m + 1)
    # min over the two halves equals the full join (exactly: same per-cell ops)
    assert np.array_equal(np.minimum(a, b), full)


def _ref_or_skip(flavour="ieee"):
    if not RefOracle.available(flavour):
        pytest.skip("reference sources not built in this environment")
    return RefOracle(flavour)


def test_block_kernel_restatement_vs_reference_sources(oracle):
    ref = _ref_or_skip()
    rng = np.random.default_rng(3)
    for trial in range(6):
        n = int(rng.integers(200, 600))
        m = int(rng.integers(4, 40))
        x = np.cumsum(rng.standard_normal(n + 1))  # +1: the kernel reads one past the windows
        PL = n - m + 1
        muS, sInv = ref.window_stats(x[:n], m)
        muS = np.concatenate([muS, np.zeros(8)])
        sInv = np.concatenate([sInv, np.zeros(8)])
        d0 = int(rng.integers(m // 4 + 1, PL // 2))
        B = int(rng.choice([1, 3, 4, 7, 64, 500]))
        T = PL - d0
        res = []
        for impl in (oracle, ref):
            prof = np.full(PL, -1.0)
            idx = np.zeros(PL, dtype=np.int64)
            qt = np.array([np.dot(x[d0 + k: d0 + k + m], x[:m]) for k in range(B)]) if B <= T \
                else np.array([np.dot(x[d0 + k: d0 + k + m], x[:m]) if d0 + k + m <= n else 0.0
                               for k in range(B)])
            qt = qt.copy()
            impl.eval_diag_block_triangle(prof, idx, prof[d0:], idx[d0:], qt, B, T, x, x[d0:], m,
                                          sInv, muS, sInv[d0:], muS[d0:], d0, 0)
            res.append((prof, idx, qt))
        assert np.array_equal(res[0][0], res[1][0]), trial
        assert np.array_equal(res[0][1], res[1][1]), trial
        assert np.array_equal(res[0][2], res[1][2]), trial


def test_restatement_vs_reference_sources_random(oracle):
    ref = _ref_or_skip()
    rng = np.random.default_rng(11)
    for trial in range(5):
        n = int(rng.integers(300, 3000))
        m = int(rng.integers(4, 120))
        x = np.cumsum(rng.standard_normal(n)) * float(rng.choice([1.0, 50.0]))
        B = int(rng.choice([7, 100, 500]))
        d2a, ia = oracle.selfjoin(x, m, blocklen=B)
        d2b, ib, _ = ref.vert_blocked(x, m, blocklen=B, shuffle=False)
        assert np.array_equal(d2a, d2b), trial
        assert np.array_equal(ia, ib), trial


def _check_cell_scores(oracle, x, m, B, d2, ix):
    PL = x.size - m + 1
    i = np.arange(PL)
    ok = d2 < 2.0 * m + 2.0  # windows some cell improved
    s = oracle.cell_scores(x, m, np.minimum(i, ix)[ok], np.maximum(i, ix)[ok], blocklen=B)
    assert ok.any()
    assert np.array_equal(2.0 * m - 2.0 * s, d2[ok])


def test_cell_scores_reproduce_profile_values(oracle):
    """A window's profile value is the score of the cell its index names, so
    recomputing that one cell in the reference's arithmetic must give the
    value bit for bit -- also for series far from zero, where the recurrence's
    rounding dominates."""
    rng = np.random.default_rng(17)
    for trial in range(4):
        n = int(rng.integers(500, 4000))
        m = int(rng.integers(8, 100))
        x = np.cumsum(rng.standard_normal(n)) * float(rng.choice([1.0, 200.0]))
        x += float(rng.choice([0.0, 1e4]))
        B = int(rng.choice([5, 64, 500]))
        d2, ix = oracle.selfjoin(x, m, blocklen=B)
        _check_cell_scores(oracle, x, m, B, d2, ix)


def test_cell_scores_vs_reference_sources(oracle):
    ref = _ref_or_skip()
    rng = np.random.default_rng(19)
    for trial in range(4):
        n = int(rng.integers(500, 4000))
        m = int(rng.integers(8, 100))
        x = np.cumsum(rng.standard_normal(n)) + float(rng.choice([0.0, 1e4]))
        B = int(rng.choice([5, 64, 500]))
        d2, ix, _ = ref.vert_blocked(x, m, blocklen=B, shuffle=True)
        _check_cell_scores(oracle, x, m, B, d2, ix)
