"""Batched joins (one persistent, graph-captured launch for many series):
every series' profile equals its standalone FP32 join with the same K --
the same alone as in the mix -- and stays within 1e-4 of the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

import thesiscode_b200 as mp
from thesiscode_b200 import workloads

pytestmark = pytest.mark.gpu


def _mix(seed, count):
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(300), np.log(30000), count))).astype(np.int64)
    ms = rng.choice([8, 16, 64, 128, 256], size=count)
    ms = np.minimum(ms, lens // 3)
    ks = rng.choice([64, 256, 1024], size=count)
    xs = [np.cumsum(rng.standard_normal(int(n))).astype(np.float32) for n in lens]
    return xs, ms, ks


def test_batch_equals_standalone_joins(gpu_ctx, oracle):
    xs, ms, ks = _mix(1, 24)
    b = mp.Batch(gpu_ctx, [x.size for x in xs], ms, ks, input_f32=True)
    res = b.run(xs)
    assert b.launch_count == 6
    for x, m, k, p in zip(xs, ms, ks, res):
        alone = gpu_ctx.selfjoin(x.astype(np.float64), int(m), precision=mp.FP32_REANCHOR,
                                 reanchor_k=int(k))
        assert np.array_equal(p.dist2, alone.dist2)
        assert np.array_equal(p.index, alone.index)
        d2, _ = oracle.selfjoin(x.astype(np.float64), int(m))
        rel = np.abs(np.sqrt(np.abs(p.dist2)) - np.sqrt(d2)) / np.sqrt(d2)
        assert rel.max() <= 1e-4, (x.size, m, k, rel.max())
    # replaying the captured graph gives the same results
    again = b.run(xs)
    for p, q in zip(res, again):
        assert np.array_equal(p.dist2, q.dist2) and np.array_equal(p.index, q.index)
    b.close()


def test_batch_float64_input_and_flat_series(gpu_ctx):
    x1 = workloads.random_walk(5000, 3)
    x2 = workloads.random_walk(4000, 4)
    x2[1000:1300] = 0.0
    b = mp.Batch(gpu_ctx, [x1.size, x2.size], [50, 64], [1024, 1024], input_f32=False)
    r = b.run([x1, x2])
    for x, m, p in zip([x1, x2], [50, 64], r):
        alone = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=1024)
        assert np.array_equal(p.dist2, alone.dist2) and np.array_equal(p.index, alone.index)
    flat = np.array([np.all(x2[i:i + 64] == x2[i]) for i in range(x2.size - 63)])
    assert np.all(r[1].dist2[flat] == 2 * 64 + 2)
    b.close()


def test_batch_rejects_bad_plans(gpu_ctx):
    with pytest.raises(mp.MpError):
        mp.Batch(gpu_ctx, [100, 50], [20, 60], [1024, 1024])
