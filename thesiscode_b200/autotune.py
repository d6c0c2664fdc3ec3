"""Autotuner for the FP32 tile shape of batched joins.

The tile of the FP32 kernel is 256 diagonals by K columns, K being also the
re-anchor interval.  Long K amortises the FP64 anchor (m FMAs per diagonal
per tile); short K cuts the empty triangle area of short series' tiles and
spreads small joins over more warps.  The tuner times single joins of seeded
random walks for each (window length, length bucket) over the candidate Ks
(all of them keep the error within 1e-4; see the accuracy tests) and stores
the fastest in a JSON table; ``lookup`` reads it, falling back to 1024.

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
    t = load()
    return int(t.get(f"{nearest_window(m)}:{bucket(n)}", 1024))


def tune(out: str = DEFAULT_TABLE, windows=WINDOWS, buckets=BUCKETS, repeats: int = 2,
         budget_s: float = 240.0) -> dict:
    import thesiscode_b200 as mp
    from thesiscode_b200 import workloads
    table = {}
    t_start = time.time()
    with mp.Context(0) as ctx:
        ctx.set_phase_timing(True)
        for m in windows:
            for b in buckets:
                n = int(1.5 * 2 ** b)
                if n < 2 * m or time.time() - t_start > budget_s:
                    continue
                x = workloads.random_walk(n, 1000 + b)
                best = None
                for K in CANDIDATES:
                    ts = []
                    for _ in range(repeats):
                        ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=K)
                        ts.append(ctx.last_phase_ms()[1])
                    t = min(ts)
                    if best is None or t < best[1]:
                        best = (K, t)
                table[f"{m}:{b}"] = best[0]
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
