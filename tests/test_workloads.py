"""Host logic on CPU: the seeded workload generators the measurements are
taken on (c3 stress layout, c4 batch, c5 request stream) and the autotuner's
table lookup used by batched joins."""
from __future__ import annotations

import json

import numpy as np
import pytest

from thesiscode_b200 import autotune, workloads


def test_random_walk_is_seeded():
    a = workloads.random_walk(1000, 7)
    assert np.array_equal(a, workloads.random_walk(1000, 7))
    assert not np.array_equal(a, workloads.random_walk(1000, 8))
    assert np.allclose(np.diff(a), np.random.default_rng(7).standard_normal(1000)[1:])


@pytest.mark.parametrize("zero", [False, True])
def test_c3_layout(zero):
    m = 128
    n = 48 * 1500
    x, mm, info = workloads.c3(n=n, m=m, zero_level=zero)
    plain = workloads.random_walk(n, 2)
    assert mm == m and x.size == n
    assert sum(k == "motif" for k, _, _ in info) == 32
    assert sum(k == "flat" for k, _, _ in info) == 16
    spans = sorted((s, s + L) for _, s, L in info)
    for (_, e0), (s1, _) in zip(spans, spans[1:]):
        assert e0 <= s1  # segments never overlap
    assert spans[0][0] >= 0 and spans[-1][1] <= n
    for kind, s, L in info:
        seg = x[s:s + L]
        if kind == "flat":
            assert L == 2 * m
            assert np.all(seg == (0.0 if zero else seg[0]))
        else:
            assert L == m
            assert not np.allclose(seg, plain[s:s + L])
    # outside the planted segments the series is the plain walk
    mask = np.ones(n, dtype=bool)
    for _, s, L in info:
        mask[s:s + L] = False
    assert np.array_equal(x[mask], plain[mask])


def test_c4_distribution():
    data = workloads.c4(count=300)
    assert len(data) == 300
    lens = np.array([s.size for s, _ in data])
    ms = {m for _, m in data}
    assert lens.min() >= 2048 and lens.max() <= 262_144
    assert ms <= {64, 128, 256} and len(ms) == 3
    assert all(s.dtype == np.float32 for s, _ in data)
    # log-uniform: the median length is near the geometric mean of the bounds
    assert 0.6 * np.sqrt(2048 * 262_144) < np.median(lens) < 1.6 * np.sqrt(2048 * 262_144)
    again = workloads.c4(count=300)
    assert all(np.array_equal(a[0], b[0]) and a[1] == b[1] for a, b in zip(data, again))


def test_c5_stream_is_poisson_and_bounded():
    rate, dur = 200.0, 10.0
    reqs = workloads.c5_stream(rate, dur)
    t = np.array([r[0] for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] < dur
    k = len(reqs)
    assert abs(k - rate * dur) < 5 * np.sqrt(rate * dur)
    for _, n, m, seed in reqs:
        assert m in (32, 64, 128, 256, 512, 1024)
        assert max(1024, 2 * m) <= n <= 1_048_576
        assert 0 <= seed < 2**31 - 1
    assert reqs == workloads.c5_stream(rate, dur)


def test_autotune_lookup(tmp_path, monkeypatch):
    assert autotune.bucket(2048) == 11 and autotune.bucket(4095) == 11 and autotune.bucket(4096) == 12
    assert autotune.bucket(10) == autotune.BUCKETS[0]
    assert autotune.bucket(1 << 30) == autotune.BUCKETS[-1]
    assert autotune.nearest_window(100) == 128 and autotune.nearest_window(90) == 64
    assert autotune.nearest_window(5000) == 1024
    table = tmp_path / "t.json"
    table.write_text(json.dumps({"128:14": 256, "64:11": 128}))
    monkeypatch.setenv("MPGPU_AUTOTUNE_TABLE", str(table))
    assert autotune.lookup(20_000, 128) == 256
    assert autotune.lookup(3_000, 60) == 128
    assert autotune.lookup(3_000, 1024) == 1024  # not in the table: the default
    monkeypatch.setenv("MPGPU_AUTOTUNE_TABLE", str(tmp_path / "missing.json"))
    assert autotune.lookup(20_000, 128) == 1024
    # entries with their measured error (the current format)
    table2 = tmp_path / "t2.json"
    table2.write_text(json.dumps({"_bound": 1e-4, "128:14": {"K": 512, "max_rel_err": 3e-5,
                                                             "join_ms": 1.0,
                                                             "within_bound": True}}))
    monkeypatch.setenv("MPGPU_AUTOTUNE_TABLE", str(table2))
    assert autotune.lookup(20_000, 128) == 512


def test_autotune_choice_is_gated_on_error():
    # the fastest candidate whose measured error is within the bound (with margin)
    trials = [(1024, 1.0, 1.2e-4), (512, 1.5, 7e-5), (256, 2.0, 5e-5), (128, 3.0, 4e-5)]
    e = autotune.choose(trials)
    assert e["K"] == 512 and e["within_bound"] and e["max_rel_err"] == 7e-5
    # nothing within the bound: the most accurate one, flagged
    e = autotune.choose([(1024, 1.0, 3e-4), (256, 2.0, 1.5e-4)])
    assert e["K"] == 256 and not e["within_bound"]
    # margin: 9e-5 is inside 1e-4 but not inside 0.8e-4
    assert autotune.choose([(1024, 1.0, 9e-5), (128, 4.0, 1e-5)])["K"] == 128


def test_committed_autotune_table_is_complete():
    t = json.load(open(autotune.DEFAULT_TABLE))
    for key, e in t.items():
        if key.startswith("_"):
            continue
        m, b = key.split(":")
        assert int(m) in autotune.WINDOWS and int(b) in autotune.BUCKETS
        K = e["K"] if isinstance(e, dict) else e
        assert K in autotune.CANDIDATES
        if isinstance(e, dict):
            # an entry is within the bound, or the most accurate candidate was kept
            assert e["within_bound"] == (e["max_rel_err"] <= autotune.SAFETY * autotune.ERROR_BOUND)
