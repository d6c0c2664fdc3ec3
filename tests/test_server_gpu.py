"""Continuous-batching server: results are identical alone and in the mix
(requests admitted while others run, overlapping on the device) and equal to
mp_selfjoin's, a small request that arrives while a large one runs finishes
first, a free slot goes to the smallest waiting request but none waits more than
about 2 s for one, admission respects
the memory budget, oversized requests are rejected; the FP64 and guarded
worker modes give mp_selfjoin's results from pool-lent scratch."""
from __future__ import annotations

import time

import numpy as np
import pytest

import thesiscode_b200 as mp
from thesiscode_b200 import workloads

pytestmark = pytest.mark.gpu


def _requests(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(60000))))
        m = int(rng.choice([32, 64, 128, 256]))
        out.append((workloads.random_walk(n, 100 + i), m))
    return out


def test_same_result_alone_and_in_the_mix(oracle):
    reqs = _requests(7, 6)
    others = _requests(8, 10)
    srv = mp.Server(0, 8 << 30, slots=4)
    alone = []
    for x, m in reqs:
        t, rc = srv.submit(x, m)
        assert rc == mp.MP_OK
        rc, p, lat, _ = srv.collect(t)
        assert rc == mp.MP_OK and lat > 0
        alone.append(p)
    # now interleaved with other traffic, all submitted at once
    tickets = []
    for i in range(max(len(reqs), len(others))):
        if i < len(others):
            tickets.append(("o", srv.submit(*others[i])[0]))
        if i < len(reqs):
            tickets.append(("r", srv.submit(*reqs[i])[0]))
    mixed = [srv.collect(t)[1] for kind, t in tickets if kind == "r"]
    # the other requests' profiles stay resident (and counted) until collected
    assert srv.stats()["bytes_in_use"] > 0
    for kind, t in tickets:
        if kind == "o":
            assert srv.collect(t, want_profile=False)[0] == mp.MP_OK
    ctx = mp.Context(0)
    for a, b, (x, m) in zip(alone, mixed, reqs):
        assert np.array_equal(a.dist2, b.dist2) and np.array_equal(a.index, b.index)
        want = ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=1024)
        assert np.array_equal(a.dist2, want.dist2) and np.array_equal(a.index, want.index)
        d2, _ = oracle.selfjoin(x, m)
        rel = np.abs(np.sqrt(np.abs(b.dist2)) - np.sqrt(d2)) / np.sqrt(d2)
        assert rel.max() <= 1e-4
    ctx.close()
    st = srv.stats()
    assert st["completed"] == len(reqs) * 2 + len(others) and st["bytes_in_use"] == 0
    srv.close()


def test_small_request_overtakes_a_large_one():
    """Requests share the device epoch by epoch: a small request submitted while
    a large one is running finishes long before it, with the same profile as
    when it runs alone."""
    big, m_big = workloads.random_walk(1_048_576, 11), 128
    small, m_small = workloads.random_walk(20_000, 12), 64
    srv = mp.Server(0, 8 << 30, slots=4)
    t_alone, _ = srv.submit(small, m_small)
    alone = srv.collect(t_alone)[1]
    t0 = time.perf_counter()
    tb, rc = srv.submit(big, m_big)
    assert rc == mp.MP_OK
    time.sleep(0.03)  # the large join is on the device now
    assert not srv.done(tb)
    ts, rc = srv.submit(small, m_small)
    dt = time.perf_counter() - t0
    assert rc == mp.MP_OK
    rs = srv.collect(ts)
    assert not srv.done(tb), "the large request finished before the small one"
    rb = srv.collect(tb, want_profile=False)
    assert rs[0] == mp.MP_OK and rb[0] == mp.MP_OK
    # finish times, both measured from the large request's submission
    assert dt + rs[2] < 0.5 * rb[2], (dt, rs[2], rb[2])
    assert np.array_equal(rs[1].dist2, alone.dist2) and np.array_equal(rs[1].index, alone.index)
    srv.close()


def test_free_slot_goes_to_the_smallest_waiting_request():
    """With its one slot taken, the server admits the waiting request with the
    fewest cells first, not the oldest: a small request submitted after a
    medium one starts (and finishes) before it."""
    big = workloads.random_walk(1_048_576, 21)
    mid = workloads.random_walk(300_000, 22)
    small = workloads.random_walk(20_000, 23)
    srv = mp.Server(0, 8 << 30, slots=1)
    tb, rc = srv.submit(big, 128)
    assert rc == mp.MP_OK
    tm, rc = srv.submit(mid, 128)
    assert rc == mp.MP_OK
    ts, rc = srv.submit(small, 64)
    assert rc == mp.MP_OK
    assert not srv.done(tb)
    rb = srv.collect(tb, want_profile=False)
    rm = srv.collect(tm, want_profile=False)
    rs = srv.collect(ts)
    assert rb[0] == rm[0] == rs[0] == mp.MP_OK
    # queue time = submission to start; the small one was submitted last
    assert rs[3] < rm[3], (rs[3], rm[3])
    assert rs[2] < rm[2], (rs[2], rm[2])
    srv.close()


def test_waiting_request_goes_first_after_two_seconds():
    """Shortest-first admission does not starve a larger request: with one
    slot and small requests always waiting beside it (each would be admitted
    before it), a medium request is admitted once it has waited 2 s."""
    small, m_small = workloads.random_walk(20_000, 41), 64
    mid, m_mid = workloads.random_walk(200_000, 42), 128
    srv = mp.Server(0, 8 << 30, slots=1)
    tickets = [srv.submit(small, m_small)[0] for _ in range(32)]
    tm, rc = srv.submit(mid, m_mid)
    assert rc == mp.MP_OK
    t0 = time.perf_counter()
    while not srv.done(tm) and time.perf_counter() - t0 < 4.0:
        if srv.stats()["waiting"] < 32:  # keep small requests queued beside it
            tickets.append(srv.submit(small, m_small)[0])
        else:
            time.sleep(0.0002)
    rm = srv.collect(tm, want_profile=False)
    rs = [srv.collect(t, want_profile=False) for t in tickets]
    assert rm[0] == mp.MP_OK and all(r[0] == mp.MP_OK for r in rs)
    # queue time = submission to start: its 2 s mark plus at most a small request
    assert 2.0 <= rm[3] < 2.5, rm[3]
    assert len(tickets) > 64  # small requests kept being admitted before it until then
    srv.close()


@pytest.mark.parametrize("prec", [mp.FP64, mp.FP32_GUARDED])
def test_worker_mode_results_and_budget(prec):
    """FP64 and guarded servers run whole mp_selfjoin calls on worker threads,
    each lent its scratch from the server's pool: results equal mp_selfjoin's,
    a budget with room for about one request at a time completes them all, and
    nothing stays counted once every result is collected."""
    m = 128
    xs = [workloads.random_walk(n, 30 + k) for k, n in enumerate((40_000, 60_000, 50_000))]
    lib = mp.load_library()
    need = max(lib.mp_selfjoin_scratch_bytes(x.size, m, prec) + 16 * (x.size - m + 1) + 512
               for x in xs)
    srv = mp.Server(0, int(need * 1.3), slots=2, precision=prec, reanchor_k=512)
    ts = []
    for x in xs:
        t, rc = srv.submit(x, m)
        assert rc == mp.MP_OK
        ts.append(t)
    res = [srv.collect(t) for t in ts]
    ctx = mp.Context(0)
    for x, r in zip(xs, res):
        assert r[0] == mp.MP_OK
        want = ctx.selfjoin(x, m, precision=prec, reanchor_k=512)
        assert np.array_equal(r[1].dist2, want.dist2) and np.array_equal(r[1].index, want.index)
    ctx.close()
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


def test_admission_by_memory_budget():
    x = workloads.random_walk(200_000, 1)
    need = mp.load_library().mp_selfjoin_scratch_bytes(x.size, 128, mp.FP32_REANCHOR)
    srv = mp.Server(0, int(need * 1.2) + (16 << 20), slots=4)  # room for one at a time
    ts = [srv.submit(x, 128)[0] for _ in range(3)]
    st = srv.stats()
    assert st["running"] <= 1 and st["waiting"] + st["running"] + st["completed"] >= 1
    res = [srv.collect(t) for t in ts]
    assert all(r[0] == mp.MP_OK for r in res)
    assert np.array_equal(res[0][1].dist2, res[2][1].dist2)
    # a request larger than the whole budget is rejected at submission
    big = workloads.random_walk(2_000_000, 2)
    t, rc = srv.submit(big, 256)
    assert rc == mp.MP_ERR_BUDGET
    assert srv.collect(t, want_profile=False)[0] == mp.MP_ERR_BUDGET
    assert srv.stats()["rejected"] == 1
    srv.close()
