"""Full search (pg_search): gaps, records and PRP accounting against GMP and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _job(pg, g, **kw):
    return pg.Job(g["P"], g["d"], g["sl"], g["max_prime"], max_m_inc=g["m_inc"],
                  max_m=g["m_start"] + g["m_inc"], **kw)


@pytest.mark.parametrize("form", [0, 1])
def test_P337_full_window(pg, form):
    """P=337, d=2310, m in [1e7, 1e7+1e4), SL 7500, primes <= 1e8: every gap equals GMP's."""
    g = golden("gaps_P337_d2310.json")
    with _job(pg, g) as job:
        assert job.k_log == g["k_log"]
        res = job.search(g["m_start"], g["m_inc"], form)
        assert [int(m) for m in res.ms] == g["ms"]
        assert list(res.prev_gap) == g["prev_gap"]
        assert list(res.next_gap) == g["next_gap"]
        assert job.records(res, g["min_merit"]) == g["records"]
        st = res.stats
        assert st["m_count"] == 2079 and st["prp_tests"] > 2 * 2079
        if form == 1:
            assert st["passes"] > 10


@pytest.mark.parametrize("name", ["gaps_P503_d2190.json", "gaps_P907_d210.json"])
def test_config_windows_against_gmp(pg, name):
    """The whole P=503 (primes <= 2e9) / P=907 (primes <= 1e10) windows; the GMP-sampled m must match."""
    g = golden(name)
    with _job(pg, g) as job:
        res = job.search(g["m_start"], g["m_inc"])
    pos = {int(m): i for i, m in enumerate(res.ms)}
    for m, a, b in zip(g["ms"], g["prev_gap"], g["next_gap"]):
        i = pos[m]
        assert (int(res.prev_gap[i]), int(res.next_gap[i])) == (a, b), m
    assert (res.prev_gap > 0).all() and (res.next_gap > 0).all()
    assert (res.prev_gap % 2 == 0).all() and (res.next_gap % 2 == 0).all()


def test_P503_sieve_matches_oracle_on_a_sample(pg, oracle):
    g = golden("gaps_P503_d2190.json")
    with _job(pg, g) as job:
        ms, rows = job.sieve_interval(g["m_start"], 400)
    with oracle.Job(g["P"], g["d"], g["sl"], g["max_prime"]) as oj:
        sel = np.arange(0, len(ms), 13)
        want = oj.sieve_m(ms[sel])
    assert np.array_equal(rows[sel], want)


def test_plain_equals_persistent(pg):
    with pg.Job(503, 2190, 10_000, 50_000_000, max_m_inc=20_000, max_m=2_000_000) as job:
        a = job.search(1_000_000, 20_000, pg.PG_SEARCH_PERSISTENT)
        b = job.search(1_000_000, 20_000, pg.PG_SEARCH_PLAIN)
    assert np.array_equal(a.prev_gap, b.prev_gap) and np.array_equal(a.next_gap, b.next_gap)
    assert b.stats["passes"] > a.stats["passes"]


@pytest.mark.parametrize("form", [0, 1])
def test_continuation_past_sl(pg, oracle, form):
    """SL far below the typical gap: most sides continue on the device past SL."""
    m_start, m_inc = 10_000_000, 600
    with pg.Job(337, 2310, 60, 1_000_000, max_m_inc=m_inc, max_m=m_start + m_inc) as job:
        res = job.search(m_start, m_inc, form)
    with oracle.Job(337, 2310, 60, 1_000_000) as oj:
        prev, nxt = oj.gmp_gaps(res.ms)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
    assert res.stats["extended_sides"] > 0 or res.stats["relaunches"] == 0


def test_confirmation_rounds(pg, oracle):
    m_start, m_inc = 10_000_000, 1_000
    with pg.Job(337, 2310, 7_500, 5_000_000, max_m_inc=m_inc, max_m=m_start + m_inc, rounds=3) as job:
        res = job.search(m_start, m_inc)
    with oracle.Job(337, 2310, 7_500, 5_000_000) as oj:
        prev, nxt, _, _ = oj.search(res.ms, 3)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
    assert res.stats["confirm_tests"] == 2 * 2 * len(res.ms)


@pytest.mark.parametrize("form", [0, 1])
def test_record_confirmation(pg, form):
    """confirm_merit: both primes of every gap with merit above it pass 16 strong bases before the search
    returns, and no other prime is tested again.  On the P=337 window (GMP gaps) the confirmation count is
    15 extra bases x 2 sides for exactly the m whose merit exceeds the threshold; the gaps do not change."""
    g = golden("gaps_P337_d2310.json")
    thr = 8.0  # 30 of the window's 2 079 m lie above it (the top merit is 11.7)
    with _job(pg, g, confirm_merit=thr) as job:
        res = job.search(g["m_start"], g["m_inc"], form)
        assert list(res.prev_gap) == g["prev_gap"] and list(res.next_gap) == g["next_gap"]
        merits = [pg.merit(job.k_log, m, a + b) for m, a, b in zip(g["ms"], g["prev_gap"], g["next_gap"])]
        over = sum(mer > thr - 1e-6 for mer in merits)
        assert over > 3
        assert res.stats["confirm_tests"] == 15 * 2 * over
        assert job.records(res, g["min_merit"]) == g["records"]


@pytest.mark.parametrize("tpi", [1, 8])
def test_record_confirmation_layouts(pg, oracle, tpi):
    """The same count on the one-thread and the lane-group kernels (P=503 operands), 8 bases in all."""
    m_start, m_inc, thr = 1_000_000, 3_000, 9.0  # a few dozen of the 789 m lie above it (the top is 15.2)
    with pg.Job(503, 2190, 10_000, 20_000_000, max_m_inc=m_inc, max_m=2_000_000, tpi=tpi, confirm_merit=thr,
                confirm_rounds=8) as job:
        res = job.search(m_start, m_inc)
        merits = [pg.merit(job.k_log, int(m), int(a) + int(b))
                  for m, a, b in zip(res.ms, res.prev_gap, res.next_gap)]
    with oracle.Job(503, 2190, 10_000, 20_000_000) as oj:
        prev, nxt = oj.gmp_gaps(res.ms)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
    over = sum(mer > thr - 1e-6 for mer in merits)
    assert over > 0 and res.stats["confirm_tests"] == 7 * 2 * over


def test_search_matches_oracle_search_and_test_count(pg, oracle):
    """Same survivors, same verdicts: the persistent form never tests fewer than the oracle."""
    m_start, m_inc = 1_000_000, 2_000
    with pg.Job(503, 2190, 10_000, 10_000_000, max_m_inc=m_inc, max_m=m_start + m_inc) as job:
        res = job.search(m_start, m_inc, pg.PG_SEARCH_PLAIN)
    with oracle.Job(503, 2190, 10_000, 10_000_000) as oj:
        prev, nxt, _, tests = oj.search(res.ms, 1)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
    assert res.stats["prp_tests"] == tests  # the plain form tests exactly the needed candidates


def test_odd_start_and_small_windows(pg, oracle):
    with pg.Job(151, 2310, 800, 1_000_000, max_m_inc=500, max_m=10**12) as job, \
            oracle.Job(151, 2310, 800, 1_000_000) as oj:
        for m_start, m_inc in [(956_702_000_001, 500), (1, 30), (13, 4), (3, 1), (999_999_999_999, 1)]:
            res = job.search(m_start, m_inc)
            prev, nxt = oj.gmp_gaps(res.ms)
            assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)


@pytest.mark.parametrize("flags", [0, 1, 6 << 16, (2 << 16) | (32 << 8) | 1])  # drain / warps-per-SM cap / both
def test_pipelined_windows_equal_synchronous(pg, flags):
    windows = [(1_000_000, 20_000), (1_020_000, 20_000), (1_040_000, 7_001), (1_000_000, 20_000)]
    with pg.Job(503, 2190, 10_000, 50_000_000, max_m_inc=20_000, max_m=2_000_000) as job:
        want = [job.search(a, b) for a, b in windows]
        got, pending = [], []
        for a, b in windows:
            pending.append(job.submit(a, b, pg.PG_SEARCH_PERSISTENT, flags))
            if len(pending) == pg.PG_SEARCH_SLOTS:
                got.append(job.wait(pending.pop(0)))
        while pending:
            got.append(job.wait(pending.pop(0)))
    for w, g in zip(want, got):
        assert np.array_equal(w.ms, g.ms)
        assert np.array_equal(w.prev_gap, g.prev_gap) and np.array_equal(w.next_gap, g.next_gap)


def test_slot_state_errors(pg):
    with pg.Job(337, 2310, 1_000, 1_000_000, max_m_inc=1_000, max_m=2 * 10**7) as job:
        t0 = job.submit(10_000_000, 1_000)
        t1 = job.submit(10_001_000, 1_000)
        with pytest.raises(pg.PrimeGapError):
            job.submit(10_002_000, 1_000)          # both slots hold un-waited tickets
        with pytest.raises(pg.PrimeGapError):
            job.sieve_interval(10_000_000, 1_000)  # slot 0 is busy
        job.wait(t1)
        job.wait(t0)
        with pytest.raises(pg.PrimeGapError):
            pg.lib.pg_search_wait(job._h, t0, None, None, None, None) and pg._check(-6)
        assert len(job.search(10_000_000, 1_000).ms) == pg.count_m(10_000_000, 1_000, 2310)


@pytest.mark.parametrize("tpi", [4, 8, 16])
def test_group_layout_search_equals_single_thread(pg, tpi):
    """The lane-group kernels (persistent, plain, confirmation) give the one-thread kernels' gaps."""
    base = pg.Job(503, 2190, 10_000, 20_000_000, max_m_inc=6_000, max_m=2_000_000, rounds=2)
    with base, pg.Job(503, 2190, 10_000, 20_000_000, max_m_inc=6_000, max_m=2_000_000, rounds=2, tpi=tpi) as grp:
        assert grp.info["tpi"] == tpi and base.info["tpi"] == 1
        want = base.search(1_000_000, 6_000)
        for form in (pg.PG_SEARCH_PERSISTENT, pg.PG_SEARCH_PLAIN):
            got = grp.search(1_000_000, 6_000, form)
            assert np.array_equal(want.prev_gap, got.prev_gap) and np.array_equal(want.next_gap, got.next_gap)
            assert got.stats["confirm_tests"] == want.stats["confirm_tests"]


@pytest.mark.parametrize("tpi", [4, 8, 16])
def test_group_layout_continuation_past_sl(pg, oracle, tpi):
    """SL far below the gaps on the lane-group kernels: the continuation launches and the trial division
    of extension positions give GMP's gaps."""
    m_start, m_inc = 1_000_000, 400
    with pg.Job(503, 2190, 60, 2_000_000, max_m_inc=m_inc, max_m=m_start + m_inc, tpi=tpi) as job:
        assert job.info["tpi"] == tpi
        res = job.search(m_start, m_inc)
    with oracle.Job(503, 2190, 60, 2_000_000) as oj:
        prev, nxt = oj.gmp_gaps(res.ms)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
    assert res.stats["extended_sides"] > 0


@pytest.mark.parametrize("tpi,limbs", [(0, 136), (16, 144)])
def test_P3001_against_gmp(pg, tpi, limbs):
    """P=3001, d=2190, X in [-40000, 40000], primes <= 1e10: 4 248-bit operands on lane groups of 8 x 17
    words (the automatic layout) and 16 x 9 words."""
    g = golden("gaps_P3001_d2190.json")
    with pg.Job(g["P"], g["d"], g["sl"], g["max_prime"], max_m_inc=64, max_m=g["m_start"] + g["m_inc"],
                tpi=tpi) as job:
        assert job.info["limbs"] == limbs and job.info["tpi"] == (tpi or 8)
        for m, a, b in zip(g["ms"], g["prev_gap"], g["next_gap"]):
            res = job.search(m, 1)
            assert list(res.ms) == [m]
            assert (int(res.prev_gap[0]), int(res.next_gap[0])) == (a, b), m


def test_graph_and_direct_launches_agree(pg):
    """The persistent form runs each window as one CUDA graph (updated in place for the next
    window); with PG_JOB_NO_GRAPH the same kernels are launched one by one."""
    windows = [(10_000_000, 3_000), (10_003_000, 3_000), (10_006_000, 1_999), (10_000_000, 3_000)]
    kw = dict(max_m_inc=3_000, max_m=2 * 10**7)
    with pg.Job(337, 2310, 7_500, 2_000_000, **kw) as g, \
            pg.Job(337, 2310, 7_500, 2_000_000, flags=pg.PG_JOB_NO_GRAPH, **kw) as d:
        for a, b in windows:
            rg, rd = g.search(a, b), d.search(a, b)
            assert rg.stats["graph_launches"] == 1 and rd.stats["graph_launches"] == 0
            assert np.array_equal(rg.prev_gap, rd.prev_gap) and np.array_equal(rg.next_gap, rd.next_gap)
            assert rg.stats["prp_ms"] > 0 and rg.stats["sieve_ms"] > 0


def test_autotune_picks_a_valid_faster_setting(pg, tmp_path):
    cache = tmp_path / "tune.json"
    knobs, ms = pg.autotune(337, 2310, 2_000, 5_000_000, 10_000_000, 2_000, cache=cache)
    assert ms > 0 and knobs["small_limit"] in (16384, 65536, 262144) and knobs["tpi"] in (0, 1, 4, 8)
    assert cache.exists()
    again, ms2 = pg.autotune(337, 2310, 2_000, 5_000_000, 10_000_000, 2_000, cache=cache)
    assert again == knobs and ms2 == ms  # served from the cache
    with pg.Job(337, 2310, 2_000, 5_000_000, max_m_inc=2_000, max_m=2 * 10**7, **knobs) as tuned, \
            pg.Job(337, 2310, 2_000, 5_000_000, max_m_inc=2_000, max_m=2 * 10**7) as plain:
        a, b = tuned.search(10_000_000, 2_000), plain.search(10_000_000, 2_000)
    assert np.array_equal(a.prev_gap, b.prev_gap) and np.array_equal(a.next_gap, b.next_gap)


def test_autotune_ex_sweeps_the_knobs(pg, tmp_path):
    """pg_autotune_ex times threads per number (1, 4, 8, 16 and automatic), the sieve tile bound, the PRP
    warps per SM (over more windows, the two best twice) and the window size with two windows in flight;
    the chosen setting is one of those, gives the same gaps, and is served from the cache the second time."""
    cache = tmp_path / "tune.json"
    res = pg.autotune_ex(503, 2190, 2_000, 20_000_000, 1_000_000, 6_000, windows=True, reps=2, cache=cache)
    assert res["settings"] == 5 + 2 + 6 + 2 + 2  # tpi, tile bound, caps, the two best caps again, windows
    assert res["knobs"]["tpi"] in (0, 1, 4, 8, 16) and res["knobs"]["small_limit"] in (0, 16384, 65536, 262144)
    assert res["warps_per_sm"] in (0, 4, 6, 8, 10, 12) and res["window_m"] in (6_000, 3_000, 1_500)
    assert res["m_per_sec"] > 0 and res["first_m_per_sec"] > 0
    assert pg.autotune_ex(503, 2190, 2_000, 20_000_000, 1_000_000, 6_000, windows=True, reps=2, cache=cache) == res
    knobs = {k: v for k, v in res["knobs"].items() if k in ("small_limit", "tpi")}
    with pg.Job(503, 2190, 2_000, 20_000_000, max_m_inc=6_000, max_m=2_000_000, **knobs) as tuned, \
            pg.Job(503, 2190, 2_000, 20_000_000, max_m_inc=6_000, max_m=2_000_000) as plain:
        a, b = tuned.search(1_000_000, 6_000), plain.search(1_000_000, 6_000)
    assert np.array_equal(a.prev_gap, b.prev_gap) and np.array_equal(a.next_gap, b.next_gap)


def test_repeat_is_deterministic(pg):
    with pg.Job(337, 2310, 7_500, 1_000_000, max_m_inc=3_000, max_m=2 * 10**7) as job:
        a = job.search(10_000_000, 3_000)
        b = job.search(10_000_000, 3_000)
    assert np.array_equal(a.prev_gap, b.prev_gap) and np.array_equal(a.next_gap, b.next_gap)


def _random_shapes(n: int, seed: int = 2026):
    """Seeded search shapes: P a prime in [11, 700], d an even divisor of P# made of small primes, sl, the
    sieve limit, an m range of 1-300 m starting anywhere below 1e12, the form, threads per number and
    confirmation rounds."""
    import random
    rng = random.Random(seed)
    primes = [q for q in range(11, 700) if all(q % r for r in range(2, int(q ** 0.5) + 1))]
    out = []
    while len(out) < n:
        P = rng.choice(primes)
        small = [q for q in (3, 5, 7, 11, 13) if q <= P]
        d = 2
        for q in small:
            if rng.random() < 0.5:
                d *= q
        sl = rng.choice([2, 30, 400, 2_000, 9_000])
        limit = rng.choice([10_000, 200_000, 3_000_000])
        m_inc = rng.randint(1, 300)
        m_start = rng.choice([1, rng.randint(1, 10**6), rng.randint(1, 10**12)])
        out.append((P, d, sl, limit, m_start, m_inc, rng.choice([0, 1]), rng.choice([0, 1, 4]), rng.choice([1, 1, 2])))
    return out


@pytest.mark.parametrize("shape", _random_shapes(48))
def test_random_shapes_against_gmp(pg, oracle, shape):
    """Every gap of a seeded random search shape equals GMP's (prevprime / nextprime of m*K)."""
    P, d, sl, limit, m_start, m_inc, form, tpi, rounds = shape
    K = 1
    for q in range(2, P + 1):
        if all(q % r for r in range(2, int(q ** 0.5) + 1)):
            K *= q
    K //= d
    if K <= limit + 2 * sl + 2:
        pytest.skip("K below the sieve limit")
    try:
        job = pg.Job(P, d, sl, limit, max_m_inc=m_inc, max_m=m_start + m_inc, tpi=tpi, rounds=rounds)
    except pg.PrimeGapError as e:
        if e.code != -3:
            raise
        pytest.skip(f"no compiled layout for this width with tpi={tpi}: {e}")
    with job:
        res = job.search(m_start, m_inc, form)
    assert len(res.ms) == pg.count_m(m_start, m_inc, d)
    with oracle.Job(P, d, sl, limit) as oj:
        prev, nxt = oj.gmp_gaps(res.ms)
    assert np.array_equal(res.prev_gap, prev) and np.array_equal(res.next_gap, nxt)
