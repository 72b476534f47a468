"""Strong PRP kernel (pg_prp_batch) against the oracle and the golden vectors."""
from __future__ import annotations

import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_golden_vectors(ctx, prp_vectors):
    items = prp_vectors["items"]
    nums = [int(it["n"], 16) for it in items]
    got1 = ctx.prp(nums, rounds=1)
    got4 = ctx.prp(nums, rounds=4)
    for it, a, b in zip(items, got1, got4):
        assert a == it["sprp2"], it
        assert b == it["mr4"], it


@pytest.mark.parametrize("P,d,m_lo,words", [(337, 2310, 10_000_000, 15), (503, 2190, 1_000_000, 22),
                                            (907, 210, 1_000_000, 40), (151, 2310, 956_702_000_000, 8)])
def test_candidates_of_the_configs(ctx, oracle, P, d, m_lo, words):
    rng = random.Random(P)
    with oracle.Job(P, d, 100, 1000, threads=1) as j:
        K = j.K
    nums = []
    while len(nums) < 300:
        m = m_lo + rng.randrange(0, 200_000)
        x = 2 * rng.randrange(-5000, 5000)
        n = m * K + x
        if n % 2 == 1:
            nums.append(n)
    # plus primes of the same size so both verdicts are exercised
    import sympy
    for _ in range(40):
        nums.append(int(sympy.nextprime(m_lo * K + rng.randrange(0, 10**6))))
    got = ctx.prp(nums, rounds=2)
    want = [oracle.prp(n, 2) for n in nums]
    assert list(got) == want
    assert sum(1 for w in want if w == 2) >= 40


def test_every_compiled_width(ctx, oracle):
    import sympy
    rng = random.Random(7)
    for words in (1, 2, 4, 7, 8, 12, 15, 16, 20, 22, 23, 24, 28, 32, 36, 40, 44, 48):
        bits = 32 * words
        nums = []
        for _ in range(6):
            p = int(sympy.nextprime(rng.getrandbits(bits - 1) | (1 << (bits - 2))))
            nums += [p, p * 3 if (p * 3).bit_length() <= bits else p + 2]
        got = ctx.prp(nums, rounds=1)
        assert list(got) == [oracle.prp(n, 1) for n in nums], words


@pytest.mark.parametrize("e", [1279, 2203, 2281, 3217, 4253, 4423])
def test_group_layouts_wide_numbers(ctx, oracle, e):
    """Numbers above 48 words run on lane groups: Mersenne primes 2^e - 1 (all-ones
    words stress every carry path), their neighbours, products and random odd numbers."""
    rng = random.Random(e)
    p = 2 ** e - 1
    nums = [p, p - 2, p + 2, p * 3, p * 1_000_003, 2 ** e + 1]
    nums += [rng.getrandbits(e) | (1 << (e - 1)) | 1 for _ in range(6)]
    got = ctx.prp(nums, rounds=2)
    assert list(got) == [oracle.prp(n, 2) for n in nums]
    assert got[0] == 2


def test_small_and_edge_numbers(ctx, oracle):
    nums = list(range(1, 2000))
    got = ctx.prp(nums, rounds=3)
    assert list(got) == [oracle.prp(n, 3) for n in nums]


def test_empty_batch(ctx):
    assert len(ctx.prp([], rounds=1)) == 0


def test_too_wide_is_an_error(pg, ctx):
    arr = np.ones((2, pg.PG_MAX_WORDS + 1), dtype=np.uint32)
    with pytest.raises(pg.PrimeGapError):
        ctx.prp_words(arr, 1)


def test_test_runner_shape(pg, ctx, oracle):
    """run_test(active, tests, results) of miller_rabin.h:364-408."""
    import sympy
    runner = pg.TestRunner(16, rounds=1, ctx=ctx)
    tests = [int(sympy.nextprime(10**40)), 10**40 + 1, 2**89 - 1, 2047, 3 * 5 * 7 * 11 + 2, 101]
    results = [-1] * len(tests)
    runner.run_test(4, tests, results)
    assert results[:4] == [1, 0, 1, 1]  # 2047 is a strong base-2 pseudoprime, as in the reference
    assert results[4:] == [0, 0]        # beyond `active`
    with pytest.raises(ValueError):
        runner.run_test(1, [4], [0])
    with pytest.raises(ValueError):
        runner.run_test(17, list(range(3, 37, 2)), [0] * 17)
