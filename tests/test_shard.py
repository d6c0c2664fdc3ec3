"""Diagonal sharding across ranks (the multi-GPU path) on CPU: world-size-2
gloo process groups, per-rank partial profiles from the oracle, merged by
MIN all-reduces of packed keys; the merged profile must equal the
single-process join (FP64 form) or the element-wise arg-min of the partial
profiles (FP32 form)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp

from thesiscode_b200 import shard, workloads


def test_partitions_cover_each_diagonal_once():
    for n, m, world in [(5000, 64, 2), (5000, 64, 3), (70000, 400, 8), (100, 8, 4)]:
        PL, excl = n - m + 1, m // 4
        seen = []
        for r in range(world):
            for a, b in shard.rank_ranges(n, m, r, world):
                seen.extend(range(a, b))
        assert sorted(seen) == list(range(excl + 1, PL))


def test_partition_balance_rule():
    # rank r takes partitions r and 2P-1-r: cell counts nearly equal per rank
    n, m, world = 200_000, 256, 4
    PL = n - m + 1
    loads = [sum(sum(PL - d for d in range(a, b)) for a, b in shard.rank_ranges(n, m, r, world))
             for r in range(world)]
    assert max(loads) / min(loads) < 1.01


def test_merge_prefers_smaller_distance_then_index():
    d2a = np.array([1.0, 2.0, 3.0, 5.0])
    ia = np.array([7, 8, 9, 4])
    d2b = np.array([1.0, 1.5, 4.0, 5.0])
    ib = np.array([3, 2, 1, 6])
    d2, ix = shard.merge_profiles([d2a, d2b], [ia, ib])
    assert d2.tolist() == [1.0, 1.5, 3.0, 5.0]
    assert ix.tolist() == [3, 2, 9, 4]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, m, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Oracle
        x = workloads.random_walk(n, 5)
        orc = Oracle()

        def compute(ranges):
            parts = [orc.selfjoin(x, m, diag_lo=lo, diag_hi=hi, nthreads=1) for lo, hi in ranges]
            d2, ix = shard.merge_profiles([p[0] for p in parts], [p[1] for p in parts])
            return torch.from_numpy(d2), torch.from_numpy(ix)

        d2, ix = shard.distributed_selfjoin(compute, n, m)
        q.put((rank, d2.numpy(), ix.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_sharded_join_equals_single_join(oracle, world):
    n, m = 4000, 64
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, m, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref_d2, ref_ix = oracle.selfjoin(workloads.random_walk(n, 5), m)
    for rank, d2, ix in res:
        assert np.array_equal(d2, ref_d2), rank
        assert np.array_equal(ix, ref_ix), rank


def _failing_worker(rank, world, port, bad_rank, q):
    """Rank `bad_rank`'s part raises; every rank must learn of it from the
    status exchange and raise ShardFailure, none may wait in the data
    exchange (a short process-group timeout bounds the test if one does)."""
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        n, m = 3000, 32
        x = workloads.random_walk(n, 9)

        def compute(ranges):
            if rank == bad_rank:
                raise RuntimeError("device scratch allocation failed")
            from oracle.oracle import Oracle
            parts = [Oracle().selfjoin(x, m, diag_lo=lo, diag_hi=hi, nthreads=1)
                     for lo, hi in ranges]
            d2, ix = shard.merge_profiles([p[0] for p in parts], [p[1] for p in parts])
            return torch.from_numpy(d2), torch.from_numpy(ix)

        try:
            shard.distributed_selfjoin(compute, n, m)
            q.put((rank, "returned", None))
        except shard.ShardFailure as e:
            q.put((rank, "ShardFailure", e.failed_ranks))
        except Exception as e:  # noqa: BLE001 - reported to the test
            q.put((rank, type(e).__name__, str(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bad_rank", [0, 1])
def test_failed_rank_is_reported_on_every_rank(oracle, bad_rank):
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, bad_rank, q))
             for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    assert res == [(r, "ShardFailure", [bad_rank]) for r in range(world)]
    assert all(p.exitcode == 0 for p in procs)



def _fp32_partial(seed, PL, m):
    """A synthetic FP32-form partial profile: d2 = 2m * u with u an FP32 value,
    some windows without a neighbour (2m + 2, index 0), some exact ties."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, 1.0, PL).astype(np.float32)
    u[::7] = np.float32(0.25)  # equal distances across ranks: the index decides
    d2 = 2.0 * m * u.astype(np.float64)
    ix = rng.integers(0, PL, PL).astype(np.int64)
    none = rng.random(PL) < 0.1
    d2[none], ix[none] = 2.0 * m + 2.0, 0
    return d2, ix


def test_fp32_keys_round_trip_and_order():
    m, PL = 96, 5000
    d2, ix = _fp32_partial(3, PL, m)
    # zero, below zero (u < 0 by rounding), tiny: all 2m times an FP32 value
    d2[:3] = 2.0 * m * np.array([0.0, -1e-7, 1e-30], dtype=np.float32).astype(np.float64)
    key = shard.pack_fp32_keys(torch.from_numpy(d2), torch.from_numpy(ix), m)
    back_d2, back_ix = shard.unpack_fp32_keys(key, m)
    assert np.array_equal(back_d2.numpy(), d2) and np.array_equal(back_ix.numpy(), ix)
    order = np.lexsort((ix, d2))
    assert np.all(np.diff(key.numpy()[order]) >= 0)


def _fp32_merge_worker(rank, world, port, m, PL, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d2, ix = _fp32_partial(40 + rank, PL, m)
        md, mi = shard.allreduce_profiles(torch.from_numpy(d2), torch.from_numpy(ix), m,
                                          fp32_form=True)
        q.put((rank, md.numpy(), mi.numpy()))
    finally:
        dist.destroy_process_group()


def test_gloo_fp32_allreduce_equals_argmin_merge():
    world, m, PL = 2, 128, 3000
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fp32_merge_worker, args=(r, world, port, m, PL, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = [_fp32_partial(40 + r, PL, m) for r in range(world)]
    want_d2, want_ix = shard.merge_profiles([p[0] for p in parts], [p[1] for p in parts])
    for rank, d2, ix in res:
        assert np.array_equal(d2, want_d2), rank
        assert np.array_equal(ix, want_ix), rank


def test_balance_by_cost_for_batch_replicas():
    data = workloads.c4(count=600)
    costs = [shard_cells(x.size, m) for x, m in data]
    for parts in (1, 2, 3, 8):
        groups = shard.balance_by_cost(costs, parts)
        assert sorted(i for g in groups for i in g) == list(range(len(costs)))
        assert all(g == sorted(g) for g in groups)
        loads = [sum(costs[i] for i in g) for g in groups]
        # largest-first onto the least-loaded group: loads differ by at most one job
        assert max(loads) - min(loads) <= max(costs)
        if parts > 1:
            assert max(loads) / min(loads) < 1.05
    assert shard.balance_by_cost([5.0, 5.0], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        shard.balance_by_cost([1.0], 0)


def shard_cells(n, m):
    L = max(n - m + 1 - m // 4 - 1, 0)
    return L * (L + 1) / 2
