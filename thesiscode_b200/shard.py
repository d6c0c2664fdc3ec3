"""Multi-GPU sharding of one self-join by diagonal ranges.

The reference splits the diagonals of the distance matrix into 2P near-equal
partitions and gives rank r partitions r and 2P-1-r, so every rank gets one
long and one short range (scrimppp/src/ScrimpTrivialPar.cpp:200-224, with
partitioning_1d.cpp:8-31).  Each rank computes a partial profile over its
ranges; one exchange step -- the reference's MPI_Allreduce with its
min-by-distance operator (ScrimpTrivialPar.cpp:68-108, 346-357) -- merges them.
Here the exchange is an element-wise minimum all-reduce over torch.distributed
(NCCL between GPUs, gloo in CPU tests) on keys that order like (squared
distance, neighbour index), so ties go to the smaller index and the result
does not depend on rank order:
  FP32 form  one 64-bit key per window, (ordered FP32 u = d2 / 2m) << 32 |
             neighbour: ONE all-reduce of 8 bytes per window;
  FP64 form  the ordered 64-bit image of d2, then the neighbour index among
             the ranks holding that minimum: two all-reduces of 8 bytes.
(An all-gather would move world x 16 bytes per window to every rank.)

A rank whose part fails (an error from the library, say out of device memory)
still takes every collective step: the ranks first exchange a status flag, and
if any part failed every rank raises ShardFailure naming the failed ranks, so
no rank is left waiting in the data exchange.
"""
from __future__ import annotations

from typing import Callable, Sequence


def near_equal_split(lo: int, hi: int, parts: int) -> list[tuple[int, int]]:
    """[lo, hi) cut into `parts` ranges whose sizes differ by at most one,
    larger ones first (partitioning_1d.cpp:8-31)."""
    n = hi - lo
    full = n - (n // parts) * parts
    size = n // parts + 1
    out = []
    for p in range(parts):
        first = p * size - max(p - full, 0)
        last = first + (size if p < full else size - 1)
        out.append((lo + first, lo + last))
    return out


def rank_ranges(n: int, m: int, rank: int, world: int, excl: int = -1) -> list[tuple[int, int]]:
    """Diagonal ranges [lo, hi) rank `rank` of `world` evaluates."""
    PL = n - m + 1
    excl = m // 4 if excl < 0 else excl
    lo, hi = excl + 1, PL
    if world == 1:
        return [(lo, hi)] if hi > lo else []
    parts = near_equal_split(lo, hi, 2 * world)
    mine = [parts[rank], parts[2 * world - 1 - rank]]
    return [(a, b) for a, b in mine if b > a]


def balance_by_cost(costs: Sequence[float], parts: int) -> list[list[int]]:
    """Indices of independent jobs (series of a batch) split into `parts`
    groups of nearly equal total cost, for replicas on several GPUs: largest
    job first, each onto the least-loaded group (ties: the lower group); each
    group lists its indices in ascending order.  No job is split."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * parts
    groups: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        g = min(range(parts), key=lambda k: (load[k], k))
        groups[g].append(i)
        load[g] += float(costs[i])
    return [sorted(g) for g in groups]


def merge_profiles(d2s: Sequence, idxs: Sequence):
    """Element-wise arg-min over partial profiles (numpy or torch arrays):
    smaller squared distance wins, ties go to the smaller index."""
    d2, ix = d2s[0], idxs[0]
    for d, i in zip(d2s[1:], idxs[1:]):
        better = (d < d2) | ((d == d2) & (i < ix))
        if hasattr(better, "numpy"):  # torch
            import torch
            d2 = torch.where(better, d, d2)
            ix = torch.where(better, i, ix)
        else:
            import numpy as np
            d2 = np.where(better, d, d2)
            ix = np.where(better, i, ix)
    return d2, ix


_SIGN_MAGNITUDE = 0x7FFFFFFFFFFFFFFF


def _ordered_i64(bits):
    """Monotone map of float64 bit patterns (as int64) to int64 order (an
    involution: applying it twice gives the bits back)."""
    import torch
    return torch.where(bits < 0, bits ^ _SIGN_MAGNITUDE, bits)


def pack_fp32_keys(d2, ix, m: int):
    """FP32-form profile (torch float64 d2 = 2m * u with u an FP32 value, int64
    neighbours < 2^32) -> int64 keys ordering like (d2, neighbour).  Windows
    without a neighbour (d2 = 2m + 2, index 0) get the largest key of all."""
    import torch
    u = (d2 / (2.0 * m)).to(torch.float32)
    ub = u.view(torch.int32)
    k32 = torch.where(ub < 0, ub ^ 0x7FFFFFFF, ub).to(torch.int64)
    key = (k32 << 32) | (ix & 0xFFFFFFFF)
    none = d2 >= 2.0 * m + 2.0
    return torch.where(none, torch.full_like(key, torch.iinfo(torch.int64).max), key)


def unpack_fp32_keys(key, m: int):
    import torch
    none = key == torch.iinfo(torch.int64).max
    k32 = (key >> 32).to(torch.int32)
    u = torch.where(k32 < 0, k32 ^ 0x7FFFFFFF, k32).view(torch.float32)
    d2 = 2.0 * m * u.to(torch.float64)
    ix = key & 0xFFFFFFFF
    d2 = torch.where(none, torch.full_like(d2, 2.0 * m + 2.0), d2)
    ix = torch.where(none, torch.zeros_like(ix), ix)
    return d2, ix


def allreduce_profiles(d2, ix, m: int, fp32_form: bool, group=None):
    """Merges every rank's partial profile (torch tensors) into the element-wise
    arg-min on every rank, ties to the smaller index: one MIN all-reduce of
    packed keys (FP32 form) or two (FP64 form: exact distance, then index)."""
    import torch
    import torch.distributed as dist
    if fp32_form:
        key = pack_fp32_keys(d2, ix, m)
        dist.all_reduce(key, op=dist.ReduceOp.MIN, group=group)
        return unpack_fp32_keys(key, m)
    od = _ordered_i64(d2.contiguous().view(torch.int64))
    best = od.clone()
    dist.all_reduce(best, op=dist.ReduceOp.MIN, group=group)
    cand = torch.where(od == best, ix, torch.full_like(ix, torch.iinfo(torch.int64).max))
    dist.all_reduce(cand, op=dist.ReduceOp.MIN, group=group)
    return _ordered_i64(best).view(torch.float64), cand


class ShardFailure(RuntimeError):
    """Raised on every rank when the part of a sharded join of any rank failed."""

    def __init__(self, failed_ranks):
        super().__init__(f"sharded self-join failed on rank(s) {failed_ranks}")
        self.failed_ranks = list(failed_ranks)


def _exchange_status(failed: bool, world: int, group, dist, torch):
    """Ranks whose part failed, as seen by every rank (one all-gather of a flag)."""
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device("cpu")
    flags = [torch.zeros(1, dtype=torch.int32, device=dev) for _ in range(world)]
    dist.all_gather(flags, torch.tensor([int(failed)], dtype=torch.int32, device=dev), group=group)
    return [r for r, f in enumerate(flags) if int(f.item())]


def distributed_selfjoin(compute: Callable, n: int, m: int, group=None, fp32_form: bool = False):
    """Runs this rank's diagonal ranges through `compute(ranges) -> (d2, idx)`
    (one call over the rank's list of (diag_lo, diag_hi) ranges; torch tensors
    of length PL on this rank's device), then merges across ranks with
    allreduce_profiles.  Every rank returns the full profile, or raises
    ShardFailure if any rank's part failed."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    ranges = rank_ranges(n, m, rank, world)
    error = None
    try:
        if ranges:
            d2, ix = compute(ranges)
        else:
            PL = n - m + 1
            d2 = torch.full((PL,), 2.0 * m + 2.0, dtype=torch.float64)
            ix = torch.zeros(PL, dtype=torch.int64)
    except Exception as e:  # reported to every rank below, then re-raised
        if world == 1:
            raise
        error = e
    if world == 1:
        return d2, ix
    failed = _exchange_status(error is not None, world, group, dist, torch)
    if failed:
        raise ShardFailure(failed) from error
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
        d2, ix = d2.to(dev), ix.to(dev)
    return allreduce_profiles(d2, ix, m, fp32_form, group)
