"""Serving loop (pg_server_*): requests of many shapes batched into common
search launches give the gaps each gives alone; admission under a tight
device-memory budget; request errors."""
from __future__ import annotations

import math
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (p, d, sl, max_prime, m_start, m_inc, rounds): three operand layouts, several
# sl per table set, ranges cut into several windows, confirmation rounds
MIX = [
    (337, 2310, 2_600, 5_000_000, 10_000_001, 3_000, 1),
    (503, 2190, 5_000, 5_000_000, 1_000_000, 9_000, 1),
    (337, 2310, 1_200, 5_000_000, 123_456_789, 2_500, 2),
    (907, 210, 7_000, 5_000_000, 2_000_000, 1_500, 1),
    (503, 2190, 3_000, 5_000_000, 999_000_001, 4_000, 1),
    (337, 210, 2_000, 5_000_000, 50_000_000, 700, 1),
    (503, 2190, 5_000, 5_000_000, 1_000_000, 9_000, 1),   # a repeat of an earlier request
    (907, 210, 7_000, 5_000_000, 77_777_777, 900, 3),
    (337, 2310, 60, 1_000_000, 10_000_000, 600, 1),       # sl far below the gaps: continuation
    (503, 2190, 4_000, 5_000_000, 3, 5_000, 1),           # m from 3
    (3001, 2190, 4_000, 5_000_000, 1_001, 300, 1),        # 136-word operands on lane groups
    (3001, 2190, 3_000, 5_000_000, 77_001, 200, 2),
]


def _alone(pg, p, d, sl, limit, m0, minc, rounds):
    with pg.Job(p, d, sl, limit, max_m_inc=minc, max_m=m0 + minc, rounds=rounds) as job:
        return job.search(m0, minc)


@pytest.mark.parametrize("preempt_us", [0, 1])
def test_mixed_requests_equal_alone(pg, preempt_us):
    """Each request's gaps equal its search alone, batched with the others.  The requests arrive widest
    operands first, a class every 0.3 s, so with preempt_us = 1 each narrower class stops the wider
    launches still running (the P=3001 launch runs over a second) and they resume from their queue heads
    once the narrower work is done."""
    want = [_alone(pg, *r) for r in MIX]
    with pg.Server(batch_m=6_000, window_m=4_000, max_windows=8, max_sl=8_000, preempt_us=preempt_us) as srv:
        ids = [0] * len(MIX)
        arrival = sorted(range(len(MIX)), key=lambda i: -MIX[i][0])
        for k, i in enumerate(arrival):
            if k and MIX[i][0] != MIX[arrival[k - 1]][0]:
                time.sleep(0.3)
            ids[i] = srv.submit(*MIX[i])
        got = {i: srv.wait(i) for i in reversed(ids)}
        st = srv.stats()
    for i, w in zip(ids, want):
        g = got[i]
        assert np.array_equal(g.ms, w.ms)
        assert np.array_equal(g.prev_gap, w.prev_gap) and np.array_equal(g.next_gap, w.next_gap)
        assert g.info["status"] == 0 and g.info["m_count"] == len(w.ms)
        assert g.info["done_s"] >= g.info["start_s"] >= g.info["submit_s"] >= 0
    assert st["requests_done"] == len(MIX)
    assert st["m_done"] == sum(len(w.ms) for w in want)
    assert st["windows"] > st["launches"]          # launches carried several windows
    assert st["tables_built"] == 6                 # one set per (p, d, max_prime)
    assert (st["preemptions"] > 0) == (preempt_us > 0)


def test_requests_from_threads_and_next_done(pg):
    reqs = [(337, 2310, 2_000 + 200 * k, 2_000_000, 10_000_000 + 5_000 * k, 1_000 + 300 * k, 1) for k in range(8)]
    want = [_alone(pg, *r) for r in reqs]
    with pg.Server(batch_m=2_000, window_m=1_000, max_windows=4, max_sl=4_000) as srv:
        ids = [None] * len(reqs)

        def client(k):
            p, d, sl, lim, m0, minc, rounds = reqs[k]
            ids[k] = srv.submit(p, d, sl, lim, m0, minc, rounds)

        th = [threading.Thread(target=client, args=(k,)) for k in range(len(reqs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        seen = [srv.next_done(timeout=120.0) for _ in reqs]
        assert sorted(seen) == sorted(ids)
        assert srv.next_done(timeout=0.05) is None
        for k, i in enumerate(ids):
            g = srv.wait(i)
            assert np.array_equal(g.prev_gap, want[k].prev_gap) and np.array_equal(g.next_gap, want[k].next_gap)


def _tables_estimate(limit: int, small: int = 65536) -> int:
    x = max(limit, 17)
    esz = 8 if limit >= 2**32 else 4
    return int(3 * esz * 1.26 * x / math.log(x) + 16 * min(small, limit) + (1 << 20))


def test_admission_evicts_idle_tables_under_a_budget(pg):
    kw = dict(batch_m=2_000, window_m=2_000, max_windows=4, max_sl=4_000)
    with pg.Server(**kw) as probe:
        slot_bytes = probe.stats()["resident_bytes"]
    limit = 20_000_000
    budget = slot_bytes + int(1.5 * _tables_estimate(limit))  # one table set at a time
    reqs = [(337, 2310, 3_000, limit, 10_000_000, 1_500, 1), (503, 2190, 3_000, limit, 1_000_000, 1_500, 1),
            (337, 2310, 3_000, limit, 20_000_000, 1_500, 1), (503, 2190, 3_000, limit, 2_000_000, 1_500, 1)]
    want = [_alone(pg, *r) for r in reqs]
    with pg.Server(hbm_budget=budget, **kw) as srv:
        ids = [srv.submit(p, d, sl, lim, m0, minc, rounds) for p, d, sl, lim, m0, minc, rounds in reqs]
        got = [srv.wait(i, timeout=300.0) for i in ids]
        st = srv.stats()
    for g, w in zip(got, want):
        assert np.array_equal(g.prev_gap, w.prev_gap) and np.array_equal(g.next_gap, w.next_gap)
    assert st["tables_evicted"] >= 1 and st["peak_bytes"] <= budget


def test_request_errors(pg):
    with pg.Server(batch_m=2_000, window_m=2_000, max_windows=4, max_sl=4_000) as srv:
        with pytest.raises(pg.PrimeGapError):
            srv.submit(337, 2310, 5_000, 1_000_000, 10_000_000, 100)   # sl above max_sl
        with pytest.raises(pg.PrimeGapError):
            srv.submit(338, 2310, 1_000, 1_000_000, 10_000_000, 100)   # p not prime
        with pytest.raises(pg.PrimeGapError):
            srv.submit(337, 2311, 1_000, 1_000_000, 10_000_000, 100)   # d odd
        bad = srv.submit(337, 2 * 347, 1_000, 1_000_000, 10_000_000, 100)  # 347 does not divide 337#
        ok = srv.submit(337, 2310, 1_000, 1_000_000, 10_000_000, 100)
        with pytest.raises(pg.PrimeGapError) as e:
            srv.wait(bad)
        assert e.value.code == -1
        assert len(srv.wait(ok).ms) == pg.count_m(10_000_000, 100, 2310)
        big = srv.submit(503, 2190, 4_000, 50_000_000, 1_000_000, 40_000)
        try:
            r = srv.wait(big, timeout=0.0)
            assert len(r.ms) == pg.count_m(1_000_000, 40_000, 2190)
        except pg.PrimeGapError as err:
            assert err.code == -5
            assert len(srv.wait(big).ms) == pg.count_m(1_000_000, 40_000, 2190)


def test_two_waiters_of_one_request(pg):
    """Two threads wait on the same request id through the C ABI: one receives the gaps, the other a
    PG_ERR_ARG that says the request went to another waiter; neither reads a request already returned."""
    with pg.Server(batch_m=2_000, window_m=2_000, max_windows=4, max_sl=4_000) as srv:
        rid = srv.submit(503, 2190, 3_000, 20_000_000, 1_000_000, 6_000)
        n = pg.count_m(1_000_000, 6_000, 2190)
        res = []  # (status, next gaps) per waiter

        def waiter():
            nxt = np.zeros(n, dtype=np.uint32)
            p32 = nxt.ctypes.data_as(pg.lib.pg_server_wait.argtypes[5])
            rc = pg.lib.pg_server_wait(srv._h, rid, 120.0, None, None, p32, None)
            res.append((rc, nxt))

        th = [threading.Thread(target=waiter) for _ in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert sorted(rc for rc, _ in res) == [-1, 0]
        assert all((nxt > 0).all() for rc, nxt in res if rc == 0)


def test_destroy_fails_queued_requests(pg):
    srv = pg.Server(batch_m=2_000, window_m=1_000, max_windows=2, max_sl=4_000)
    for k in range(6):
        srv.submit(503, 2190, 3_000, 20_000_000, 1_000_000 + 10_000 * k, 5_000)
    srv.close()  # finishes the launches in flight, fails the rest, frees everything


def test_request_larger_than_the_budget_fails(pg):
    kw = dict(batch_m=2_000, window_m=2_000, max_windows=4, max_sl=4_000)
    with pg.Server(**kw) as probe:
        slot_bytes = probe.stats()["resident_bytes"]
    budget = slot_bytes + int(1.5 * _tables_estimate(5_000_000))
    with pg.Server(hbm_budget=budget, **kw) as srv:
        small = srv.submit(337, 2310, 2_000, 5_000_000, 10_000_000, 500)
        huge = srv.submit(503, 2190, 2_000, 400_000_000, 1_000_000, 500)   # ~240 MB of tables
        assert len(srv.wait(small).ms) == pg.count_m(10_000_000, 500, 2310)
        with pytest.raises(pg.PrimeGapError) as e:
            srv.wait(huge, timeout=120.0)
        assert e.value.code == -4 and "exceed the budget" in str(e.value)
        assert srv.stats()["peak_bytes"] <= budget
