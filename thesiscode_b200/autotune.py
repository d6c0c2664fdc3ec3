"""Autotuner for the FP32 tile shape of batched joins.

The tile of the FP32 kernel is 256 diagonals by K columns, K being also the
re-anchor interval.  Long K amortises the FP64 anchor (m FMAs per diagonal
per tile); short K cuts the empty triangle area of short series' tiles,
spreads small joins over more warps and shortens the FP32 recurrence between
anchors (smaller rounding drift).  For each (window length, length bucket) the
tuner runs single joins of a seeded random walk with every candidate K, times
them, and measures each one's maximum relative distance error against the FP64
form on the same series (bit-identical to the reference's arithmetic).  Only
candidates within the error bound (1e-4, the FP32 form's target, less a
safety margin) are eligible; the fastest of them is stored with its measured
error.  When no candidate meets the bound the most accurate one is stored and
the entry says so.  ``lookup`` reads the table, falling back to 1024.

The error is measured on random walks; other data (planted motifs beside
constant stretches, say) can exceed it -- the guarded form covers those.

    python -m thesiscode_b200.autotune [--out thesiscode_b200/autotune_table.json]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "autotune_table.json")
CANDIDATES = (128, 256, 512, 1024)
WINDOWS = (32, 64, 128, 256, 512, 1024)
BUCKETS = tuple(range(11, 21))  # n in [2^b, 2^(b+1)): 2,048 .. 2,097,151
ERROR_BOUND = 1e-4
SAFETY = 0.8  # a candidate must measure within SAFETY * ERROR_BOUND

_table = None


def bucket(n: int) -> int:
    return min(max(int(math.log2(max(n, 2))), BUCKETS[0]), BUCKETS[-1])


def nearest_window(m: int) -> int:
    return min(WINDOWS, key=lambda w: abs(math.log2(w) - math.log2(max(m, 2))))


def load(path: str | None = None) -> dict:
    global _table
    path = path or os.environ.get("MPGPU_AUTOTUNE_TABLE", DEFAULT_TABLE)
    if _table is None or _table.get("_path") != path:
        try:
            with open(path) as f:
                _table = json.load(f)
        except (OSError, ValueError):
            _table = {}
        _table["_path"] = path
    return _table


def lookup(n: int, m: int) -> int:
    e = load().get(f"{nearest_window(m)}:{bucket(n)}", 1024)
    return int(e["K"] if isinstance(e, dict) else e)


def choose(trials: list[tuple[int, float, float]]) -> dict:
    """(K, join ms, max relative error) per candidate -> the table entry: the
    fastest candidate within SAFETY * ERROR_BOUND, else the most accurate."""
    ok = [t for t in trials if t[2] <= SAFETY * ERROR_BOUND]
    if ok:
        K, ms, err = min(ok, key=lambda t: (t[1], t[0]))
    else:
        K, ms, err = min(trials, key=lambda t: (t[2], t[1]))
    return {"K": int(K), "join_ms": round(float(ms), 4), "max_rel_err": float(err),
            "within_bound": bool(err <= SAFETY * ERROR_BOUND)}


def tune(out: str = DEFAULT_TABLE, windows=WINDOWS, buckets=BUCKETS, repeats: int = 2,
         budget_s: float = 240.0) -> dict:
    import numpy as np

    import thesiscode_b200 as mp
    from thesiscode_b200 import workloads
    table = {"_bound": ERROR_BOUND, "_safety": SAFETY, "_candidates": list(CANDIDATES)}
    t_start = time.time()
    with mp.Context(0) as ctx:
        ctx.set_phase_timing(True)
        for m in windows:
            for b in buckets:
                n = int(1.5 * 2 ** b)
                if n < 2 * m or time.time() - t_start > budget_s:
                    continue
                x = workloads.random_walk(n, 1000 + b)
                ref = np.sqrt(np.abs(ctx.selfjoin(x, m, precision=mp.FP64).dist2))
                trials = []
                for K in CANDIDATES:
                    ts = []
                    for _ in range(repeats):
                        p = ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=K)
                        ts.append(ctx.last_phase_ms()[1])
                    err = float(np.max(np.abs(np.sqrt(np.abs(p.dist2)) - ref) / ref))
                    trials.append((K, min(ts), err))
                table[f"{m}:{b}"] = choose(trials)
    with open(out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    global _table
    _table = None
    return table


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--budget-s", type=float, default=240.0)
    a = ap.parse_args()
    print(json.dumps(tune(a.out, budget_s=a.budget_s), indent=1))
