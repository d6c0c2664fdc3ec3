"""Poisson request stream against the continuous-batching server.

Replays workload c5 (arrivals at `rate` per second for `duration` seconds,
lengths log-uniform in [1024, 1048576], m uniform in {32..1024}, seed 4):
each request is submitted at its arrival time; a collector thread gathers
finished profiles.  Reports p50/p99 latency (arrival to finish), admitted
cells/s and rejections.

    python -m thesiscode_b200.serve --rate 30 --duration 10
"""
from __future__ import annotations

import argparse
import json
import threading
import time

import numpy as np

import thesiscode_b200 as mp
from thesiscode_b200 import workloads


def run_stream(rate: float, duration: float, slots: int = 4, budget_gb: float = 64.0,
               seed: int = 4, max_n: int | None = None, drain_timeout: float = 120.0):
    reqs = workloads.c5_stream(rate, duration, seed)
    if max_n:
        reqs = [(t, min(n, max_n), m, s) for t, n, m, s in reqs]
    series = {}
    srv = mp.Server(0, int(budget_gb * (1 << 30)), slots, mp.FP32_REANCHOR, 1024)
    tickets, lock = [], threading.Lock()
    lat, que, rejected = [], [], 0
    stop = threading.Event()

    def collector():
        while not (stop.is_set() and not tickets):
            with lock:
                pending = list(tickets)
            progressed = False
            for t in pending:
                if srv.done(t):
                    rc, _, l, q = srv.collect(t, want_profile=False)
                    with lock:
                        tickets.remove(t)
                    if rc == mp.MP_OK:
                        lat.append(l)
                        que.append(q)
                    progressed = True
            if not progressed:
                time.sleep(0.0005)

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    cells_submitted = 0.0
    for (ta, n, m, s) in reqs:
        x = series.get(s)
        if x is None:
            x = workloads.random_walk(n, s)
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        t, rc = srv.submit(x, m)
        if rc == mp.MP_ERR_BUDGET:
            rejected += 1
            srv.collect(t, want_profile=False)
            continue
        cells_submitted += mp.cells(n, m)
        with lock:
            tickets.append(t)
    t_sub = time.perf_counter() - t0
    stop.set()
    th.join(timeout=drain_timeout)
    t_end = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat_ms = np.array(lat) * 1e3
    return {
        "rate_hz": rate, "duration_s": duration, "requests": len(reqs), "completed": len(lat),
        "rejected": rejected, "slots": slots,
        "p50_ms": float(np.percentile(lat_ms, 50)) if lat else None,
        "p99_ms": float(np.percentile(lat_ms, 99)) if lat else None,
        "queue_p50_ms": float(np.percentile(np.array(que) * 1e3, 50)) if que else None,
        "cells_per_s": st["cells"] / t_end if t_end > 0 else None,
        "submit_window_s": t_sub, "wall_s": t_end,
    }


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, nargs="+", default=[10, 30, 100])
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=64.0)
    a = ap.parse_args()
    for r in a.rate:
        print(json.dumps(run_stream(r, a.duration, a.slots, a.budget_gb)), flush=True)
