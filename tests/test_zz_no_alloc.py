"""pg_next_prime_noalloc: the allocation-free entry point, for callers that
cannot call cudaMalloc (their device memory belongs to another allocator, or
an allocation would stall their running pipeline).

Called through the C ABI with device buffers the test owns; every result is
checked against the existing entry point pg_prp_batch (the first k whose
number + 2k passes the strong base-2 test), on consecutive calls of different
sizes, since all calls share one scratch array.  This file sorts last so a run
that stops at the first failure has already run every other test; it also
passes alone in a fresh process (the first call looks up the scratch address).
"""
from __future__ import annotations

import ctypes
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOT_FOUND = 0xFFFFFFFF


def _fn(pg):
    f = pg.lib.pg_next_prime_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _numbers(seed: int, n: int, bits: int) -> list[int]:
    rng = random.Random(seed)
    out = [rng.getrandbits(bits) | (1 << (bits - 1)) | 1 for _ in range(n)]
    out[0] = 2 ** 89 - 1 if bits > 90 else out[0]   # already prime: k = 0
    out[1] = out[1] + 1                              # even: never prime
    return out


def _expected(ctx, nums: list[int], words: int, max_steps: int) -> list[int]:
    """First k < max_steps with nums[i] + 2k passing base 2, via pg_prp_batch.
    At 48 words (the widest layout) candidates of 2^1536 or more are skipped."""
    res = []
    top = 1 << (32 * words) if words == 48 else None
    for x in nums:
        ks = [k for k in range(max_steps) if top is None or x + 2 * k < top]
        if not ks or x % 2 == 0:
            res.append(NOT_FOUND)
            continue
        cands = np.stack([np.frombuffer((x + 2 * k).to_bytes(words * 4 + 4, "little"), dtype=np.uint32)
                          for k in ks])
        passed = ctx.prp_words(cands, rounds=1)
        hit = np.nonzero(passed == 1)[0]
        res.append(ks[int(hit[0])] if len(hit) else NOT_FOUND)
    return res


def _run(pg, nums: list[int], words: int, max_steps: int) -> list[int]:
    import torch
    arr = np.stack([np.frombuffer(x.to_bytes(words * 4, "little"), dtype=np.uint32) for x in nums])
    d_in = torch.from_numpy(arr.view(np.int32).copy()).cuda()
    d_out = torch.full((len(nums),), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _fn(pg)(d_in.data_ptr(), len(nums), words, max_steps, d_out.data_ptr(), stream.cuda_stream)
    assert rc == 0, pg.lib.pg_last_error().decode()
    torch.cuda.synchronize()
    return [int(v) & 0xFFFFFFFF for v in d_out.cpu().numpy()]


def test_noalloc_matches_prp_batch_on_consecutive_calls(pg, ctx):
    cases = [(_numbers(1, 48, 700), 22, 600),    # 703-bit numbers, 22 words
             (_numbers(2, 20, 470), 15, 400),    # a smaller second call: stale entries must not leak
             (_numbers(3, 48, 700), 22, 600)]
    for nums, words, steps in cases:
        got = _run(pg, nums, words, steps)
        assert got == _expected(ctx, nums, words, steps)
        assert got[1] == NOT_FOUND
        assert any(v != NOT_FOUND for v in got)


def test_noalloc_rejects_sizes_beyond_the_scratch(pg):
    import torch
    f = _fn(pg)
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    assert f(buf.data_ptr(), 65537, 1, 4, buf.data_ptr(), None) == -1
    assert "PG_NOALLOC_MAX_N" in pg.lib.pg_last_error().decode()
    assert f(buf.data_ptr(), 1, 49, 4, buf.data_ptr(), None) == -3
    assert f(buf.data_ptr(), 0, 4, 4, buf.data_ptr(), None) == 0


def test_noalloc_full_batch_then_one_step(pg, ctx):
    """n = PG_NOALLOC_MAX_N (the queue runs to n * max_steps items), checked on
    a sample against pg_prp_batch; then a call of max_steps 1 right after it,
    on numbers whose found[] entries the big call filled."""
    n, words, steps = 65536, 22, 4
    rng = random.Random(5)
    nums = [rng.getrandbits(700) | (1 << 699) | 1 for _ in range(n)]
    got = _run(pg, nums, words, steps)
    sample = sorted(rng.sample(range(n), 96))
    assert [got[i] for i in sample] == _expected(ctx, [nums[i] for i in sample], words, steps)
    assert sum(v != NOT_FOUND for v in got) > n // 100   # ~3.6% of 4-candidate runs hold a prime
    small = nums[:64]
    got1 = _run(pg, small, words, 1)
    assert got1 == _expected(ctx, small, words, 1)


@pytest.mark.parametrize("words", [22, 48])
def test_noalloc_numbers_at_the_top_of_their_width(pg, ctx, words):
    """Numbers just below 2^(32*words): their candidates carry into a word the
    input does not have.  Below 48 words the kernel runs a layout with a spare
    word and tests them at full width (2^704 + 327 is the first prime above
    2^704); at 48 words they are skipped (no prime lies in 2^1536 - 599 ..
    2^1536, so every result is 0xFFFFFFFF)."""
    top = 1 << (32 * words)
    nums = [top - 2 * j - 1 for j in (0, 1, 5, 40, 150, 299)]
    steps = 300
    got = _run(pg, nums, words, steps)
    assert got == _expected(ctx, nums, words, steps)
    if words == 22:
        assert any(v != NOT_FOUND and nums[i] + 2 * v >= top for i, v in enumerate(got))
    else:
        assert all(v == NOT_FOUND for v in got)
