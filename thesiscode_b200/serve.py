"""Poisson request stream against the continuous-batching server.

Replays workload c5 (arrivals at `rate` per second for `duration` seconds,
lengths log-uniform in [1024, 1048576], m uniform in {32..1024}, seed 4):
each request is submitted at its arrival time; a collector thread gathers
finished profiles.  Reports p50/p99 latency from the scheduled arrival to the
finished profile, admitted cells/s and rejections.

With several servers (one per GPU, `devices`), requests go to them in turn
(round-robin replicas; requests are independent, so nothing is exchanged).

The series are generated by a producer thread a bounded number of requests
ahead of the submitter, so generating a long series does not hold back the
arrivals behind it.  If the submitter still reaches an arrival late (the
producer fell behind, or a submit took long), the lateness is added to that
request's latency, so the figure always runs from the scheduled arrival.

    python -m thesiscode_b200.serve --rate 30 --duration 10
"""
from __future__ import annotations

import argparse
import json
import queue
import threading
import time

import numpy as np

import thesiscode_b200 as mp
from thesiscode_b200 import workloads


def _producer(reqs, out: queue.Queue, stop: threading.Event):
    for (_, n, _, s) in reqs:
        x = workloads.random_walk(n, s)
        while not stop.is_set():
            try:
                out.put(x, timeout=0.1)
                break
            except queue.Full:
                continue
        if stop.is_set():
            return


def run_stream(rate: float, duration: float, slots: int = 32, budget_gb: float = 64.0,
               seed: int = 4, max_n: int | None = None, drain_timeout: float = 120.0,
               server=None, lookahead: int = 32, servers=None, devices=None):
    """Replays the c5 stream at `rate`.  Requests go round-robin to `servers`
    (objects with submit/done/collect/stats/close), or to `server`, or to new
    mp.Server replicas on `devices` (default: device 0), each admitting at most
    `slots` requests at once within `budget_gb` of device memory."""
    reqs = workloads.c5_stream(rate, duration, seed)
    if max_n:
        reqs = [(t, min(n, max_n), m, s) for t, n, m, s in reqs]
    own = servers is None and server is None
    if servers is None and server is not None:
        servers = [server]
    elif servers is None:
        servers = []
        try:
            for d in (devices if devices else [0]):
                servers.append(mp.Server(d, int(budget_gb * (1 << 30)), slots, mp.FP32_REANCHOR,
                                         1024))
        except Exception:
            for srv in servers:
                srv.close()
            raise
    servers = list(servers)
    tickets, lock = [], threading.Lock()  # (replica, ticket) pairs in flight
    late = {}  # (replica, ticket) -> seconds between the scheduled arrival and the submit
    lat, que, rejected = [], [], 0
    stop = threading.Event()

    def collector():
        while not (stop.is_set() and not tickets):
            with lock:
                pending = list(tickets)
            progressed = False
            for key in pending:
                srv, t = servers[key[0]], key[1]
                if srv.done(t):
                    rc, _, l, q = srv.collect(t, want_profile=False)
                    with lock:
                        tickets.remove(key)
                        d = late.pop(key, 0.0)
                    if rc == mp.MP_OK:
                        lat.append(l + d)
                        que.append(q + d)
                    progressed = True
            if not progressed:
                time.sleep(0.0005)

    ready: queue.Queue = queue.Queue(maxsize=max(1, lookahead))
    halt = threading.Event()
    prod = threading.Thread(target=_producer, args=(reqs, ready, halt), daemon=True)
    prod.start()
    # the first arrivals' series are generated before the clock starts
    while prod.is_alive() and ready.qsize() < min(lookahead, len(reqs)):
        time.sleep(0.001)
    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    cells_submitted = 0.0
    late_s = []
    per_replica = [0] * len(servers)
    try:
        for i, (ta, n, m, s) in enumerate(reqs):
            now = time.perf_counter() - t0
            if ta > now:
                time.sleep(ta - now)
            x = ready.get()
            d = max(0.0, time.perf_counter() - t0 - ta)
            k = i % len(servers)
            srv = servers[k]
            t, rc = srv.submit(x, m)
            late_s.append(d)
            per_replica[k] += 1
            if rc == mp.MP_ERR_BUDGET:
                rejected += 1
                srv.collect(t, want_profile=False)
                continue
            cells_submitted += mp.cells(n, m)
            with lock:
                late[(k, t)] = d
                tickets.append((k, t))
    finally:
        halt.set()
        t_sub = time.perf_counter() - t0
        stop.set()
        th.join(timeout=drain_timeout)
        t_end = time.perf_counter() - t0
        cells_done = sum(srv.stats()["cells"] for srv in servers)
        if own:
            for srv in servers:
                srv.close()
    lat_ms = np.array(lat) * 1e3
    return {
        "rate_hz": rate, "duration_s": duration, "requests": len(reqs), "completed": len(lat),
        "rejected": rejected, "slots": slots, "replicas": len(servers),
        "requests_per_replica": per_replica,
        "p50_ms": float(np.percentile(lat_ms, 50)) if lat else None,
        "p99_ms": float(np.percentile(lat_ms, 99)) if lat else None,
        "queue_p50_ms": float(np.percentile(np.array(que) * 1e3, 50)) if que else None,
        "submit_late_p99_ms": float(np.percentile(np.array(late_s) * 1e3, 99)) if late_s else None,
        "cells_per_s": cells_done / t_end if t_end > 0 else None,
        "cells_submitted": cells_submitted,
        "submit_window_s": t_sub, "wall_s": t_end,
    }


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, nargs="+", default=[10, 30, 100])
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--slots", type=int, default=32)
    ap.add_argument("--budget-gb", type=float, default=64.0)
    ap.add_argument("--gpus", type=int, default=1, help="replicas, one server per GPU")
    a = ap.parse_args()
    for r in a.rate:
        print(json.dumps(run_stream(r, a.duration, a.slots, a.budget_gb,
                                    devices=list(range(a.gpus)))), flush=True)
