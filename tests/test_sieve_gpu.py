"""Sieve kernels (pg_sieve_interval) bit for bit against the oracle."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _job(pg, P, d, sl, limit, m_start, m_inc, **kw):
    return pg.Job(P, d, sl, limit, max_m_inc=m_inc, max_m=m_start + m_inc, **kw)


def test_golden_rows(pg):
    g = golden("sieve_rows.json")
    with _job(pg, g["P"], g["d"], g["sl"], g["max_prime"], g["m_start"], g["m_inc"]) as job:
        ms, rows = job.sieve_interval(g["m_start"], g["m_inc"])
    assert [int(m) for m in ms] == g["ms"]
    assert rows.shape[1] == g["words_per_m"]
    assert [hashlib.sha256(r.tobytes()).hexdigest() for r in rows] == g["row_sha256"]


@pytest.mark.parametrize("P,d,sl,limit,m_start,m_inc,small", [
    (503, 2190, 10_000, 20_000_000, 1_000_000, 3_000, 0),        # large-prime kernel from 65536
    (503, 2190, 10_000, 20_000_000, 1_000_000, 3_000, 1_000),    # most primes in the large kernel
    (337, 2310, 7_500, 60_000, 10_000_000, 4_000, 0),            # limit below the small split
    (907, 210, 18_000, 5_000_000, 1_000_000, 1_000, 4_096),
    (907, 2190, 40_000, 3_000_000, 1, 600, 0),                   # m from 1, SL 40000, 1 244-bit K
    (151, 2310, 1_234, 1_000_000, 956_702_000_001, 5_000, 0),    # odd m_start, m above 2^32
    (337, 2310, 3, 100_000, 10_000_000, 500, 0),                 # SL = 3: one position per side
])
def test_rows_match_oracle(pg, oracle, P, d, sl, limit, m_start, m_inc, small):
    with _job(pg, P, d, sl, limit, m_start, m_inc, small_limit=small) as job:
        ms, rows = job.sieve_interval(m_start, m_inc)
    with oracle.Job(P, d, sl, limit) as oj:
        assert np.array_equal(ms, oracle.coprime_ms(m_start, m_inc, d))
        want = oj.sieve_m(ms)
    assert np.array_equal(rows, want)


@pytest.mark.parametrize("flags", [0, 1, 2, 8])  # automatic split, step every Y, modular search, compact walk table
@pytest.mark.parametrize("P,d,sl,limit,m_start,m_inc", [
    (503, 2190, 10_000, 30_000_000, 1_000_000, 4_000),
    (337, 2310, 200_000 // 2, 5_000_000, 10_000_000, 1_000),   # sly = 50 000 < small split: two hits per j
    (907, 210, 2_000, 40_000_000, 1_000_000, 20_000),
])
def test_large_prime_methods_agree(pg, oracle, flags, P, d, sl, limit, m_start, m_inc):
    with _job(pg, P, d, sl, limit, m_start, m_inc, flags=flags, small_limit=2_000) as job:
        ms, rows = job.sieve_interval(m_start, m_inc)
    with oracle.Job(P, d, sl, limit) as oj:
        want = oj.sieve_m(ms)
    assert np.array_equal(rows, want)


@pytest.mark.parametrize("P,d,sl,limit,m_start,m_inc", [
    (503, 2190, 4_000, 4_300_000_000, 1_000_000, 60),
    (211, 2310, 300, 4_400_000_000, 10**12 + 1, 60),    # m above 2^32, short rows
    # W >= 8192: single-precision quotients on the 32-bit levels; few odd m, so warps of primes
    # expecting under 1/64 hit stop their searches at the window bound, from the 64-bit levels on
    (907, 210, 18_000, 4_300_000_000, 1_000_000, 60),
    (503, 2190, 10_000, 4_300_000_000, 1_000_001, 120),
])
def test_wide_primes_above_2_32(pg, oracle, P, d, sl, limit, m_start, m_inc):
    """max_prime above 2^32: 64-bit prime tables and residues."""
    with _job(pg, P, d, sl, limit, m_start, m_inc) as job:
        ms, rows = job.sieve_interval(m_start, m_inc)
        assert job.info["num_primes"] > 200_000_000
    with oracle.Job(P, d, sl, limit) as oj:
        want = oj.sieve_m(ms)
    assert np.array_equal(rows, want)


def test_windows_reuse_one_job(pg, oracle):
    P, d, sl, limit = 337, 2310, 2_000, 2_000_000
    with pg.Job(P, d, sl, limit, max_m_inc=2_000, max_m=10**8) as job, oracle.Job(P, d, sl, limit) as oj:
        for m_start, m_inc in [(10_000_000, 2_000), (10_002_000, 1_000), (20_000_001, 7), (99_998_000, 2_000)]:
            ms, rows = job.sieve_interval(m_start, m_inc)
            assert np.array_equal(rows, oj.sieve_m(ms))


def test_window_too_large_is_an_error(pg):
    with pg.Job(337, 2310, 100, 10_000, max_m_inc=100, max_m=10**8) as job:
        with pytest.raises(pg.PrimeGapError):
            job.sieve_interval(10_000_000, 101)
        with pytest.raises(pg.PrimeGapError):
            job.sieve_interval(10**8, 100)


@pytest.mark.parametrize("bad", [dict(p=338), dict(d=15), dict(d=2 * 1009), dict(sl=1), dict(sl=300_000)])
def test_bad_jobs_are_errors(pg, bad):
    kw = dict(p=337, d=2310, sl=100, max_prime=10_000, max_m_inc=100, max_m=10**8)
    kw.update(bad)
    with pytest.raises(pg.PrimeGapError):
        pg.Job(**kw)


def _random_sieve_shapes(n: int, seed: int = 77):
    """Seeded sieve shapes: P, d (even divisor of P# of small primes), sl, limit, small-prime bound, m range."""
    import random
    rng = random.Random(seed)
    primes = [q for q in range(40, 1000) if all(q % r for r in range(2, int(q ** 0.5) + 1))]
    out = []
    for _ in range(n):
        P = rng.choice(primes)
        d = 2
        for q in (3, 5, 7, 11, 13, 73):
            if q <= P and rng.random() < 0.4:
                d *= q
        sl = rng.choice([2, 7, 64, 1_000, 5_000, 30_000])
        limit = rng.choice([5_000, 100_000, 2_000_000, 30_000_000])
        small = rng.choice([0, 2_000, 20_000, 200_000])
        m_inc = rng.randint(1, 2_000)
        m_start = rng.choice([1, rng.randint(1, 10**7), rng.randint(1, 10**13)])
        out.append((P, d, sl, limit, small, m_start, m_inc))
    return out


@pytest.mark.parametrize("shape", _random_sieve_shapes(20))
def test_random_sieve_rows(pg, oracle, shape):
    """Every bit of every row of a seeded random sieve shape equals the oracle's."""
    P, d, sl, limit, small, m_start, m_inc = shape
    with _job(pg, P, d, sl, limit, m_start, m_inc, small_limit=small) as job:
        ms, rows = job.sieve_interval(m_start, m_inc)
    with oracle.Job(P, d, sl, limit) as oj:
        assert np.array_equal(ms, oracle.coprime_ms(m_start, m_inc, d))
        want = oj.sieve_m(ms)
    assert np.array_equal(rows, want)


@pytest.mark.parametrize("P,d,sl,limit,small,m_start,m_inc", [
    (503, 2190, 10_000, 20_000_000, 1_000, 1_000_000, 50_000),   # p from 10 007: 256 segments of 98 odd m
    (907, 210, 2_000, 8_000_000, 2_000, 1_000_000, 40_000),      # p from 4 001: 64 segments
    (337, 2310, 64, 3_000_000, 0, 10_000_000, 60_000),           # sl 64: walks of width 65
])
def test_segmented_large_prime_rows(pg, oracle, P, d, sl, limit, small, m_start, m_inc):
    """Primes that expect many hits per window are sieved by (prime, segment of m) threads from walk
    constants computed once per job; sampled rows of a wide window equal the oracle's, and a second, smaller
    window on the same job (fewer segments per prime) too."""
    with _job(pg, P, d, sl, limit, m_start, m_inc, small_limit=small) as job, oracle.Job(P, d, sl, limit) as oj:
        for start, inc in [(m_start, m_inc), (m_start + 999, m_inc // 7)]:
            ms, rows = job.sieve_interval(start, inc)
            sel = np.arange(0, len(ms), 53)
            assert np.array_equal(rows[sel], oj.sieve_m(ms[sel]))


@pytest.mark.parametrize("P,d,sl,limit,small,m_start,m_inc", [
    (503, 2190, 30_000, 60_000_000, 0, 1_000_000, 24),          # bound from p > 64 * 12 * 30 001 = 2.3e7
    (337, 2310, 9_000, 200_000_000, 0, 10_000_000, 40),         # W = 9 000: single-precision quotients
    (151, 2310, 20_000, 100_000_000, 2_000, 10**12 + 1, 16),    # m above 2^32
])
def test_bounded_search_rows(pg, oracle, P, d, sl, limit, small, m_start, m_inc):
    """Windows of a few odd m and wide rows: warps whose primes all expect under 1/64 hit stop each
    modular search once it provably lands past the window, and the 32-bit levels take their quotients from
    a rounded-down single-precision reciprocal (W >= 8192); every row equals the oracle's."""
    with _job(pg, P, d, sl, limit, m_start, m_inc, small_limit=small) as job:
        ms, rows = job.sieve_interval(m_start, m_inc)
    with oracle.Job(P, d, sl, limit) as oj:
        want = oj.sieve_m(ms)
    assert len(ms) > 0 and np.array_equal(rows, want)
