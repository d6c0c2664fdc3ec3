"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's golden vectors.

FP64 form: profile values must be BIT-IDENTICAL to the reference (IEEE
build); indices identical except where the two neighbours tie in the
reference's own arithmetic -- their cell scores, recomputed by the oracle with
the reference's per-cell operations, give distances within 1e-9 relative.
Which of two such candidates the reference keeps depends on its shuffled block
order; the GPU keeps the smaller index among candidates whose squared
distances agree to the index key's resolution (~1e-10 relative).
FP32 re-anchored form: distances within 1e-4 relative of the FP64 oracle;
indices point to a neighbour whose exact distance is within 1e-4 of the best.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import thesiscode_b200 as mp
from thesiscode_b200 import workloads

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4  # max relative error of the distance, FP32 re-anchored form


def check_fp64_indices(oracle, x, m, d2, idx, ref_idx, blocklen=500):
    diff = np.nonzero(idx != ref_idx)[0]
    if diff.size:
        a, b = idx[diff], ref_idx[diff]
        stats = oracle.window_stats(x, m)
        sa = oracle.cell_scores(x, m, np.minimum(diff, a), np.maximum(diff, a), blocklen,
                                stats=stats)
        sb = oracle.cell_scores(x, m, np.minimum(diff, b), np.maximum(diff, b), blocklen,
                                stats=stats)
        da = np.sqrt(np.abs(2.0 * m - 2.0 * sa))
        db = np.sqrt(np.abs(2.0 * m - 2.0 * sb))
        tie = (sa == sb) | (np.abs(da - db) <= 1e-9 * db)
        assert tie.all(), list(zip(diff[~tie][:5], a[~tie][:5], b[~tie][:5], da[~tie][:5],
                                   db[~tie][:5]))
    return diff.size


@pytest.mark.parametrize("m", [16, 64, 400])
def test_fp64_test_ascii_bit_identical(gpu_ctx, oracle, golden_ascii, m):
    x = golden_ascii["series"]
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    assert np.array_equal(p.dist2, golden_ascii[f"d2_m{m}"])
    assert check_fp64_indices(oracle, x, m, p.dist2, p.index, golden_ascii[f"idx_m{m}"]) == 0


def test_fp64_stats_and_first_qt_bit_identical(gpu_ctx, golden_ascii):
    x = golden_ascii["series"]
    muS, sInv = gpu_ctx.window_stats(x, 64)
    assert np.array_equal(muS, golden_ascii["muS_m64"])
    assert np.array_equal(sInv, golden_ascii["sInv_m64"])
    qt = gpu_ctx.first_qt(x, 64, 0, 2000)
    assert np.array_equal(qt, golden_ascii["qt_m64_0_2000"])


def test_fp64_edge_cases(gpu_ctx, oracle, golden_edges):
    for name, c in golden_edges.items():
        m, B = (int(v) for v in c["meta"])
        p = gpu_ctx.selfjoin(c["x"], m, precision=mp.FP64, blocklen=B)
        assert np.array_equal(p.dist2, c["d2"], equal_nan=True), name
        check_fp64_indices(oracle, c["x"], m, p.dist2, p.index, c["idx"], blocklen=B)


def test_fp64_c1_digest(gpu_ctx, digests):
    x, m = workloads.c1()
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    assert hashlib.sha256(p.dist2.tobytes()).hexdigest() == digests["c1"]["d2_sha256"]
    assert hashlib.sha256(p.index.tobytes()).hexdigest() == digests["c1"]["idx_sha256"]


def test_fp64_c2_digest(gpu_ctx, digests):
    if "c2" not in digests:
        pytest.skip("c2 digest not recorded")
    x, m = workloads.c2()
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    assert hashlib.sha256(p.dist2.tobytes()).hexdigest() == digests["c2"]["d2_sha256"]


def test_fp64_random_sizes_vs_oracle(gpu_ctx, oracle):
    rng = np.random.default_rng(5)
    for trial in range(8):
        n = int(rng.integers(64, 20000))
        m = int(rng.integers(4, min(300, n // 2)))
        B = int(rng.choice([1, 5, 64, 500, 1000]))
        x = np.cumsum(rng.standard_normal(n)) * float(rng.choice([1.0, 30.0]))
        d2, idx = oracle.selfjoin(x, m, blocklen=B)
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP64, blocklen=B)
        assert np.array_equal(p.dist2, d2), (trial, n, m, B)
        check_fp64_indices(oracle, x, m, p.dist2, p.index, idx, blocklen=B)


def test_fp64_diagonal_range(gpu_ctx, oracle):
    x = workloads.random_walk(12000, 9)
    m = 100
    for lo, hi in [(26, 1000), (1000, 5000), (5000, 11901), (26, 27), (11900, 11901)]:
        d2, idx = oracle.selfjoin(x, m, diag_lo=lo, diag_hi=hi)
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
        assert np.array_equal(p.dist2, d2), (lo, hi)
        check_fp64_indices(oracle, x, m, p.dist2, p.index, idx)


def flat_dense_series(n=16000, m=32, every=200, seed=12):
    """Random walk with a constant segment of 2m samples (held at the walk's
    value, so the windows' variance rounds to 0 or below and sInv is inf or
    NaN) every `every` samples."""
    x = workloads.random_walk(n, seed)
    for s in range(50, n - 2 * m, every):
        x[s:s + 2 * m] = x[s]
    return x, m


@pytest.mark.parametrize("width", [100, 300, 1000, 3000])
def test_fp64_nan_cells_beside_valid_cells(gpu_ctx, oracle, width):
    """NaN cells of constant windows never select, and never hide the valid
    cell beside them in a lane's R diagonals (band widths 100..3000 give
    R = 1, 2, 4, 8), in full bands and in a range's partial last band."""
    x, m = flat_dense_series()
    PL = x.size - m + 1
    for lo in (m // 4 + 1, PL // 3, PL - width):
        hi = min(lo + width, PL)
        d2, idx = oracle.selfjoin(x, m, diag_lo=lo, diag_hi=hi)
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
        assert np.array_equal(p.dist2, d2, equal_nan=True), (width, lo, hi)
        check_fp64_indices(oracle, x, m, p.dist2, p.index, idx)


def test_fp64_device_pointers_match_host(gpu_ctx):
    import torch
    x = workloads.random_walk(30000, 4)
    m = 128
    ph = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
    xd = torch.from_numpy(x).cuda()
    d2 = torch.empty(x.size - m + 1, dtype=torch.float64, device="cuda")
    ix = torch.empty(x.size - m + 1, dtype=torch.int64, device="cuda")
    gpu_ctx.selfjoin(xd, m, precision=mp.FP64, out=(d2, ix))
    assert np.array_equal(d2.cpu().numpy(), ph.dist2)
    assert np.array_equal(ix.cpu().numpy(), ph.index)


def test_block_interface_vs_oracle(gpu_ctx, oracle):
    """mp_eval_diag_block_triangle with the reference kernel's contract:
    aliased (self-join) and disjoint (tile) profile views, carried tmpQ."""
    rng = np.random.default_rng(21)
    for trial in range(6):
        n = int(rng.integers(300, 4000))
        m = int(rng.integers(4, 64))
        x = np.cumsum(rng.standard_normal(n + 1))
        PL = n - m + 1
        muS, sInv = oracle.window_stats(x[:n], m)
        muS = np.concatenate([muS, np.zeros(8)])
        sInv = np.concatenate([sInv, np.zeros(8)])
        d0 = int(rng.integers(m // 4 + 1, PL // 2))
        B = int(rng.choice([1, 3, 8, 100, 500]))
        T = PL - d0
        qt0 = np.array([np.dot(x[d0 + k: d0 + k + m], x[:m]) if d0 + k + m <= n else 0.0
                        for k in range(B)])
        res = []
        for impl in ("oracle", "gpu"):
            prof = np.full(PL, -1.0)
            prof[::7] = 0.5  # pre-existing scores, as after earlier blocks
            idx = np.zeros(PL, dtype=np.int64)
            idx[::7] = 3
            qt = qt0.copy()
            args = (prof, idx, prof[d0:], idx[d0:], qt, B, T, x, x[d0:], m, sInv, muS, sInv[d0:],
                    muS[d0:], d0, 0)
            if impl == "oracle":
                oracle.eval_diag_block_triangle(*args)
            else:
                gpu_ctx.eval_diag_block_triangle(*args)
            res.append((prof, idx, qt))
        assert np.array_equal(res[0][0], res[1][0]), trial
        assert np.array_equal(res[0][2][:min(B, T)], res[1][2][:min(B, T)]), trial
        assert (res[0][1] != res[1][1]).sum() == 0, trial


def test_block_interface_disjoint_tile(gpu_ctx, oracle):
    rng = np.random.default_rng(8)
    m, T, B = 32, 900, 200
    xa = np.cumsum(rng.standard_normal(T + m + 1))
    xb = np.cumsum(rng.standard_normal(T + m + 1))
    mua, sa = oracle.window_stats(xa, m)
    mub, sb = oracle.window_stats(xb, m)
    qt0 = np.array([np.dot(xb[k:k + m], xa[:m]) for k in range(B)])
    res = []
    for impl in ("oracle", "gpu"):
        pc, ic = np.full(T + m, -1.0), np.full(T + m, -1, dtype=np.int64)
        pr, ir = np.full(T + m, -1.0), np.full(T + m, -1, dtype=np.int64)
        qt = qt0.copy()
        args = (pc, ic, pr, ir, qt, B, T, xa, xb, m, sa, mua, sb, mub, 5000, 7000)
        (oracle if impl == "oracle" else gpu_ctx).eval_diag_block_triangle(*args)
        res.append((pc, ic, pr, ir, qt))
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("K", [64, 256, 1024])
def test_fp32_reanchor_error_c1(gpu_ctx, oracle, K):
    x, m = workloads.c1()
    d2, idx = oracle.selfjoin(x, m)
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=K)
    dt = np.sqrt(d2)
    dg = np.sqrt(np.abs(p.dist2))
    rel = np.abs(dg - dt) / dt
    assert rel.max() <= FP32_TOL, rel.max()
    # the chosen neighbour is (near-)optimal: its exact distance is within tol
    bad = np.nonzero(p.index != idx)[0]
    for i in bad[:200]:
        a = np.sqrt(oracle.pair_d2(x, m, i, p.index[i]))
        assert a <= dt[i] * (1 + FP32_TOL) + 1e-12, (i, a, dt[i])


def test_fp32_flat_windows_follow_reference_convention(gpu_ctx, oracle, golden_edges):
    c = golden_edges["flat_zero_level"]
    m = int(c["meta"][0])
    x = c["x"]
    p = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR)
    flat = np.array([np.all(x[i:i + m] == x[i]) for i in range(x.size - m + 1)])
    assert np.all(p.dist2[flat] == 2 * m + 2) and np.all(p.index[flat] == 0)
    assert not np.any(flat[p.index[~flat]])
    ok = ~flat
    rel = np.abs(np.sqrt(p.dist2[ok]) - np.sqrt(c["d2"][ok])) / np.sqrt(c["d2"][ok])
    assert rel.max() <= FP32_TOL


def test_fp32_random_sizes(gpu_ctx, oracle):
    rng = np.random.default_rng(17)
    for trial in range(6):
        n = int(rng.integers(100, 30000))
        m = int(rng.integers(8, min(400, n // 2)))
        x = np.cumsum(rng.standard_normal(n))
        d2, _ = oracle.selfjoin(x, m)
        K = int(rng.choice([64, 256, 1024]))
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=K)
        rel = np.abs(np.sqrt(np.abs(p.dist2)) - np.sqrt(d2)) / np.sqrt(d2)
        assert rel.max() <= FP32_TOL, (trial, n, m, K, rel.max())


def test_errors_are_status_codes(gpu_ctx):
    x = workloads.random_walk(100, 1)
    with pytest.raises(mp.MpError) as e:
        gpu_ctx.selfjoin(x, 200)
    assert e.value.status == mp.MP_ERR_INVALID_ARG
    small = mp.Context(0, mem_budget_bytes=1 << 16)
    with pytest.raises(mp.MpError) as e:
        small.selfjoin(workloads.random_walk(100000, 1), 64)
    assert e.value.status == mp.MP_ERR_BUDGET
    small.close()


def test_selfjoin_ranges_one_call_equals_separate_calls(gpu_ctx, oracle):
    """A rank's two diagonal partitions (the reference's triv_par rule) in one
    mp_selfjoin_ranges call give the element-wise arg-min of the two separate
    joins; the FP64 form stays bit-identical to the oracle on those ranges."""
    from thesiscode_b200 import shard
    x = workloads.random_walk(20000, 31)
    m = 64
    for rank in (0, 1):
        ranges = shard.rank_ranges(x.size, m, rank, 2)
        assert len(ranges) == 2
        for prec in (mp.FP64, mp.FP32_REANCHOR):
            one = gpu_ctx.selfjoin_ranges(x, m, ranges, precision=prec, reanchor_k=256)
            parts = [gpu_ctx.selfjoin(x, m, precision=prec, reanchor_k=256, diag_lo=a, diag_hi=b)
                     for a, b in ranges]
            md, mi = shard.merge_profiles([p.dist2 for p in parts], [p.index for p in parts])
            assert np.array_equal(one.dist2, md), (rank, prec)
            if prec == mp.FP32_REANCHOR:
                assert np.array_equal(one.index, mi), rank
            else:
                refs = [oracle.selfjoin(x, m, diag_lo=a, diag_hi=b) for a, b in ranges]
                rd, ri = shard.merge_profiles([r[0] for r in refs], [r[1] for r in refs])
                assert np.array_equal(one.dist2, rd), rank
                check_fp64_indices(oracle, x, m, one.dist2, one.index, ri)
    with pytest.raises(mp.MpError) as e:
        gpu_ctx.selfjoin_ranges(x, m, shard.rank_ranges(x.size, m, 0, 2),
                                precision=mp.FP32_GUARDED)
    assert e.value.status == mp.MP_ERR_NOT_SUPPORTED


def test_fp64_exact_repeats_keep_reference_values_and_tie_rule(gpu_ctx, oracle):
    """A series made of exact repeats of one pattern (plus a drifting copy), so
    that many cells share the same score: the threshold-pruned selection must
    still give the reference's values bit for bit and neighbours that tie with
    the reference's in its own arithmetic."""
    rng = np.random.default_rng(77)
    pattern = np.cumsum(rng.standard_normal(300))
    x = np.concatenate([pattern, pattern, pattern + 5.0, pattern, pattern * 2.0, pattern])
    for m in (32, 100):
        d2, idx = oracle.selfjoin(x, m)
        p = gpu_ctx.selfjoin(x, m, precision=mp.FP64)
        assert np.array_equal(p.dist2, d2), m
        check_fp64_indices(oracle, x, m, p.dist2, p.index, idx)
