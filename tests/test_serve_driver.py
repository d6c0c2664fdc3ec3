"""The serving driver (thesiscode_b200/serve.py) on CPU, against a fake server
with a fixed service time: every request of the c5 stream is submitted and
collected, rejections are counted, and latency runs from the scheduled arrival
(lateness of the submitter included)."""
from __future__ import annotations

import threading
import time

import thesiscode_b200 as mp
from thesiscode_b200 import serve, workloads


class FakeServer:
    """Finishes a request `service_s` after its submit; rejects series longer
    than `max_len`; each submit takes `submit_s`."""

    def __init__(self, service_s=0.002, max_len=None, submit_s=0.0):
        self.service_s, self.max_len, self.submit_s = service_s, max_len, submit_s
        self.reqs, self.next, self.cells = {}, 1, 0.0
        self.lock = threading.Lock()

    def submit(self, x, m):
        if self.submit_s:
            time.sleep(self.submit_s)
        with self.lock:
            t = self.next
            self.next += 1
            rejected = self.max_len is not None and x.size > self.max_len
            self.reqs[t] = (time.perf_counter(), x.size, m, rejected)
        return t, (mp.MP_ERR_BUDGET if rejected else mp.MP_OK)

    def done(self, t):
        with self.lock:
            t0, _, _, rejected = self.reqs[t]
        return rejected or time.perf_counter() >= t0 + self.service_s

    def collect(self, t, want_profile=True):
        while not self.done(t):
            time.sleep(0.0002)
        with self.lock:
            _, n, m, rejected = self.reqs.pop(t)
            if rejected:
                return mp.MP_ERR_BUDGET, None, 0.0, 0.0
            self.cells += mp.cells(n, m)
        return mp.MP_OK, None, self.service_s, 0.0

    def stats(self):
        return {"cells": self.cells}


def test_every_request_is_submitted_and_collected():
    fake = FakeServer(service_s=0.003)
    r = serve.run_stream(100.0, 1.0, server=fake, max_n=20_000)
    reqs = workloads.c5_stream(100.0, 1.0)
    assert r["requests"] == len(reqs) and r["completed"] == len(reqs) and r["rejected"] == 0
    assert not fake.reqs  # nothing left uncollected
    want = sum(mp.cells(min(n, 20_000), m) for _, n, m, _ in reqs)
    assert r["cells_submitted"] == want and fake.cells == want
    assert r["p50_ms"] >= 3.0 and r["p99_ms"] < 200.0
    assert r["submit_late_p99_ms"] < 100.0


def test_rejections_are_counted_not_collected_as_results():
    fake = FakeServer(max_len=8_000)
    r = serve.run_stream(100.0, 1.0, server=fake, max_n=20_000)
    reqs = workloads.c5_stream(100.0, 1.0)
    big = sum(min(n, 20_000) > 8_000 for _, n, _, _ in reqs)
    assert 0 < big < len(reqs)
    assert r["rejected"] == big and r["completed"] == len(reqs) - big


def test_latency_counts_a_late_submitter():
    # each submit takes 20 ms against arrivals ~5 ms apart: later requests are
    # submitted ever later, and their latency must include that delay
    fake = FakeServer(service_s=0.001, submit_s=0.02)
    r = serve.run_stream(200.0, 0.4, server=fake, max_n=4_000)
    n = r["requests"]
    assert n > 40
    # the last submit happens ~n * 20 ms after the start, its arrival at <= 0.4 s
    assert r["submit_late_p99_ms"] > 0.5 * (n * 20.0 - 400.0)
    assert r["p99_ms"] >= r["submit_late_p99_ms"] * 0.9


def test_replicas_take_requests_in_turn():
    fakes = [FakeServer(service_s=0.002), FakeServer(service_s=0.002)]
    r = serve.run_stream(100.0, 1.0, servers=fakes, max_n=20_000)
    n = r["requests"]
    assert r["replicas"] == 2 and r["requests_per_replica"] == [(n + 1) // 2, n // 2]
    assert r["completed"] == n and not fakes[0].reqs and not fakes[1].reqs
    reqs = workloads.c5_stream(100.0, 1.0)
    want = [sum(mp.cells(min(nn, 20_000), m) for i, (_, nn, m, _) in enumerate(reqs) if i % 2 == k)
            for k in range(2)]
    assert [f.cells for f in fakes] == want
