"""ctypes wrapper of the CPU oracle (oracle/oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, the smoke check in __graft_entry__.py and bench.py's CPU-baseline
and reference legs import this module.  The product library never does.

The oracle restates the reference's CPU path (see oracle.c's header for the
file:line of every function it follows) on top of the GMP runtime.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "liboracle.so"


def build(force: bool = False) -> pathlib.Path:
    """Compile liboracle.so with the committed Makefile."""
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, u32, u64, i32, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_size_t
        P32, P64 = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)
        L.or_job_create.restype = vp
        L.or_job_create.argtypes = [u32, u32, u32, u64, i32, ctypes.POINTER(ctypes.c_int)]
        L.or_job_free.argtypes = [vp]
        L.or_job_K_log.restype = ctypes.c_double
        L.or_job_K_log.argtypes = [vp]
        L.or_job_num_sieve_primes.restype = sz
        L.or_job_num_sieve_primes.argtypes = [vp]
        L.or_job_K_words.restype = i32
        L.or_job_K_words.argtypes = [vp, P32, i32]
        L.or_coprime_ms.restype = sz
        L.or_coprime_ms.argtypes = [u64, u64, u32, P64, sz]
        L.or_words_per_m.restype = u32
        L.or_words_per_m.argtypes = [u32]
        L.or_sieve_m.argtypes = [vp, P64, sz, P32, i32]
        L.or_sieve_x.restype = sz
        L.or_sieve_x.argtypes = [vp, u64, u64, u32, u32, P32, i32]
        L.or_prp.restype = i32
        L.or_prp.argtypes = [P32, i32, i32]
        L.or_probab_prime.restype = i32
        L.or_probab_prime.argtypes = [P32, i32, i32]
        L.or_candidate_words.restype = i32
        L.or_candidate_words.argtypes = [vp, u64, ctypes.c_int64, P32, i32]
        L.or_search.restype = u64
        L.or_search.argtypes = [vp, P64, sz, i32, P32, P32, P32, i32]
        L.or_gmp_gaps.argtypes = [vp, P64, sz, P32, P32, i32]
        L.or_sieve_x_rows.restype = sz
        L.or_sieve_x_rows.argtypes = [vp, u64, u64, ctypes.POINTER(ctypes.c_int64), sz, P32, i32]
        L.or_prp_batch.argtypes = [P32, sz, i32, i32, ctypes.POINTER(ctypes.c_int32), i32]
        L.or_primes.restype = P64
        L.or_primes.argtypes = [u64, u64, ctypes.POINTER(sz), i32]
        L.or_gmp_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _p32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _p64(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


def int_to_words(n: int, nwords: int | None = None) -> np.ndarray:
    if nwords is None:
        nwords = max(1, (n.bit_length() + 31) // 32)
    return np.frombuffer(n.to_bytes(nwords * 4, "little"), dtype=np.uint32).copy()


def words_to_int(w) -> int:
    return int.from_bytes(np.asarray(w, dtype=np.uint32).tobytes(), "little")


def prp(n: int, rounds: int = 1) -> int:
    """Number of strong-PRP bases (2, 3, 5, ...) passed, as miller_rabin.h:216-248."""
    w = int_to_words(n)
    return lib().or_prp(_p32(w), len(w), rounds)


def prp_batch(numbers, rounds: int = 1, threads: int | None = None) -> np.ndarray:
    """prp() of many numbers on `threads` host threads."""
    numbers = [int(x) for x in numbers]
    nw = max(1, max((x.bit_length() + 31) // 32 for x in numbers))
    arr = np.ascontiguousarray(np.stack([int_to_words(x, nw) for x in numbers]))
    out = np.zeros(len(numbers), dtype=np.int32)
    lib().or_prp_batch(_p32(arr), len(numbers), nw, rounds, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                       threads or default_threads())
    return out


def probab_prime(n: int, reps: int = 25) -> int:
    """GMP mpz_probab_prime_p (0 composite, 1 probable prime, 2 prime)."""
    w = int_to_words(n)
    return lib().or_probab_prime(_p32(w), len(w), reps)


def primes(lo: int, hi: int, threads: int | None = None) -> np.ndarray:
    n = ctypes.c_size_t(0)
    ptr = lib().or_primes(lo, hi, ctypes.byref(n), threads or default_threads())
    out = np.ctypeslib.as_array(ptr, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint64)
    ctypes.CDLL(None).free(ctypes.cast(ptr, ctypes.c_void_p))
    return out


def coprime_ms(m_start: int, m_inc: int, d: int) -> np.ndarray:
    n = lib().or_coprime_ms(m_start, m_inc, d, None, 0)
    out = np.zeros(n, dtype=np.uint64)
    lib().or_coprime_ms(m_start, m_inc, d, _p64(out), n)
    return out


def words_per_m(sl: int) -> int:
    return lib().or_words_per_m(sl)


class Job:
    """K = P#/d plus the sieve tables for primes <= limit (gap_common.cpp:60-65,
    gap_search_gpu.cpp:471-501)."""

    ERRORS = {-1: "d does not divide P#", -2: "K <= 1", -3: "d must be even",
              -4: "P is not prime", -5: "K too small for the sieve limit"}

    def __init__(self, P: int, d: int, sl: int, limit: int, threads: int | None = None):
        self.P, self.d, self.sl, self.limit = P, d, sl, limit
        self.sly = sl // 2
        self.threads = threads or default_threads()
        err = ctypes.c_int(0)
        self._h = lib().or_job_create(P, d, sl, limit, self.threads, ctypes.byref(err))
        if not self._h:
            raise ValueError(self.ERRORS.get(err.value, f"oracle error {err.value}"))
        nw = lib().or_job_K_words(self._h, None, 0)
        kw = np.zeros(nw, dtype=np.uint32)
        lib().or_job_K_words(self._h, _p32(kw), nw)
        self.K_words = kw
        self.K = words_to_int(kw)
        self.K_log = lib().or_job_K_log(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().or_job_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def num_sieve_primes(self) -> int:
        return lib().or_job_num_sieve_primes(self._h)

    def sieve_m(self, ms) -> np.ndarray:
        ms = np.ascontiguousarray(ms, dtype=np.uint64)
        W = words_per_m(self.sl)
        out = np.zeros((len(ms), W), dtype=np.uint32)
        lib().or_sieve_m(self._h, _p64(ms), len(ms), _p32(out), self.threads)
        return out

    def sieve_x(self, m_start: int, m_inc: int, w_lo: int = 0, w_hi: int = 2**32 - 1) -> np.ndarray:
        W = words_per_m(self.sl)
        n = len(coprime_ms(m_start, m_inc, self.d))
        out = np.zeros((n, W), dtype=np.uint32)
        lib().or_sieve_x(self._h, m_start, m_inc, w_lo, w_hi, _p32(out), self.threads)
        return out

    def sieve_x_rows(self, m_start: int, m_inc: int, ys) -> np.ndarray:
        """The reference's per-X sieve for the rows Y in ys only (others stay 0)."""
        ys = np.ascontiguousarray(ys, dtype=np.int64)
        W = words_per_m(self.sl)
        n = len(coprime_ms(m_start, m_inc, self.d))
        out = np.zeros((n, W), dtype=np.uint32)
        lib().or_sieve_x_rows(self._h, m_start, m_inc, ys.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                              len(ys), _p32(out), self.threads)
        return out

    def search(self, ms, rounds: int = 1):
        """(prev_gap, next_gap, overflow_mask, prp_tests) for every m."""
        ms = np.ascontiguousarray(ms, dtype=np.uint64)
        prev = np.zeros(len(ms), dtype=np.uint32)
        nxt = np.zeros(len(ms), dtype=np.uint32)
        ovf = np.zeros(len(ms), dtype=np.uint32)
        tests = lib().or_search(self._h, _p64(ms), len(ms), rounds, _p32(prev), _p32(nxt), _p32(ovf), self.threads)
        return prev, nxt, ovf, int(tests)

    def gmp_gaps(self, ms):
        """Ground truth: mpz_prevprime / mpz_nextprime from m*K."""
        ms = np.ascontiguousarray(ms, dtype=np.uint64)
        prev = np.zeros(len(ms), dtype=np.uint32)
        nxt = np.zeros(len(ms), dtype=np.uint32)
        lib().or_gmp_gaps(self._h, _p64(ms), len(ms), _p32(prev), _p32(nxt), self.threads)
        return prev, nxt

    def candidate(self, m: int, X: int) -> int:
        return m * self.K + X


def gmp_version() -> str:
    return lib().or_gmp_version().decode()
