"""prime-gap-gpu_b200: B200 prime-gap search behind the C ABI of libprimegap.so.

Python mirror of the reference's interfaces for the hot path:

  TestRunner(n, rounds).run_test(active, tests, results)
      test_runner_t<params> (miller_rabin.h:296-409): strong PRP of a batch,
      results[i] = 1 if tests[i] passed every base, 0 otherwise.
  Job(p, d, sl, max_prime, ...)
      K = P#/d and the sieve tables (init_K gap_common.cpp:60-65, the sieve
      prework gap_search_gpu.cpp:471-501), resident on the device.
  Job.sieve_interval(m_start, m_inc)
      the per-m sieve rows (sieve_interval_cpu's contract, both signs of X).
  Job.search(m_start, m_inc, form)
      previous/next prime gap of every m coprime to d, found on the device
      (the GPU batches of gpu_testing.cu:203-350 plus the CPU overflow
      finishing of overflow.cpp:145-188).
  merit(), format_record(), records()
      overflow.cpp:162-188.
  Server(device).submit(p, d, sl, max_prime, m_start, m_inc) / wait(id)
      many such searches from any thread, batched continuously on one device
      (no counterpart in the reference, which runs one search per process).

There is no CPU fallback: importing this package loads libprimegap.so and
raises if it is missing or was built without the symbols declared in
include/primegap.h.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "build" / "libprimegap.so"

PG_OK = 0
PG_SEARCH_PERSISTENT = 0
PG_SEARCH_PLAIN = 1
PG_MAX_WORDS = 160
PG_JOB_LARGE_STEP = 0x1
PG_JOB_LARGE_SEARCH = 0x2
PG_JOB_NO_GRAPH = 0x4
PG_JOB_COMPACT_WALK = 0x8

# every symbol include/primegap.h declares
EXPORTS = (
    "pg_ctx_create", "pg_ctx_destroy", "pg_ctx_stream", "pg_last_error", "pg_version", "pg_measure_imad_peak",
    "pg_prp_batch", "pg_prp_batch_device",
    "pg_job_create", "pg_job_destroy", "pg_job_get_info", "pg_job_k_words",
    "pg_count_m", "pg_sieve_interval", "pg_search", "pg_merit", "pg_format_record", "pg_next_prime_noalloc",
    "pg_search_submit", "pg_search_wait", "pg_job_stream", "pg_autotune", "pg_autotune_ex",
    "pg_server_create", "pg_server_submit", "pg_server_wait", "pg_server_next_done", "pg_server_get_stats",
    "pg_server_clock", "pg_server_destroy",
)
PG_SEARCH_SLOTS = 2
PG_SUBMIT_DRAIN = 0x1


def PG_SUBMIT_DRAIN_LANES(d: int) -> int:
    return (d & 0xff) << 8


def PG_SUBMIT_WARPS_PER_SM(w: int) -> int:
    return (w & 0xff) << 16


class PrimeGapError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libprimegap error {code}: {msg}")
        self.code = code


class JobParams(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_uint32), ("d", ctypes.c_uint32), ("sl", ctypes.c_uint32),
        ("max_prime", ctypes.c_uint64), ("max_m_inc", ctypes.c_uint64), ("max_m", ctypes.c_uint64),
        ("rounds", ctypes.c_uint32), ("small_limit", ctypes.c_uint32),
        ("ext_window", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("search_hits", ctypes.c_uint32),
        ("tpi", ctypes.c_uint32), ("confirm_merit", ctypes.c_double), ("confirm_rounds", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]


class JobInfo(ctypes.Structure):
    _fields_ = [
        ("k_bits", ctypes.c_uint32), ("limbs", ctypes.c_uint32), ("tpi", ctypes.c_uint32),
        ("words_per_m", ctypes.c_uint32),
        ("side_capacity", ctypes.c_uint32), ("num_primes", ctypes.c_uint64), ("num_small", ctypes.c_uint64),
        ("k_log", ctypes.c_double), ("setup_seconds", ctypes.c_double), ("device_bytes", ctypes.c_uint64),
    ]


class SearchStats(ctypes.Structure):
    _fields_ = [
        ("m_count", ctypes.c_uint64), ("prp_tests", ctypes.c_uint64), ("confirm_tests", ctypes.c_uint64),
        ("extended_sides", ctypes.c_uint64), ("passes", ctypes.c_uint32), ("relaunches", ctypes.c_uint32),
        ("sieve_ms", ctypes.c_double), ("prp_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
        ("search_kernel_ms", ctypes.c_double), ("kernel_launches", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("graph_launches", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("survivors", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("params", JobParams), ("warps_per_sm", ctypes.c_uint32), ("settings", ctypes.c_uint32),
        ("window_m", ctypes.c_uint64), ("m_per_sec", ctypes.c_double), ("first_m_per_sec", ctypes.c_double),
    ]


PG_TUNE_WINDOW = 0x1


class ServerParams(ctypes.Structure):
    _fields_ = [
        ("hbm_budget", ctypes.c_uint64), ("batch_m", ctypes.c_uint32), ("window_m", ctypes.c_uint32),
        ("max_windows", ctypes.c_uint32), ("max_sl", ctypes.c_uint32), ("small_limit", ctypes.c_uint32),
        ("ext_window", ctypes.c_uint32), ("tpi", ctypes.c_uint32), ("warps_per_sm", ctypes.c_uint32),
        ("slots", ctypes.c_uint32), ("preempt_us", ctypes.c_uint32),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_uint32), ("d", ctypes.c_uint32), ("sl", ctypes.c_uint32), ("rounds", ctypes.c_uint32),
        ("max_prime", ctypes.c_uint64), ("m_start", ctypes.c_uint64), ("m_inc", ctypes.c_uint64),
    ]


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("m_count", ctypes.c_uint64), ("k_log", ctypes.c_double), ("submit_s", ctypes.c_double),
        ("start_s", ctypes.c_double), ("done_s", ctypes.c_double), ("windows", ctypes.c_uint32),
        ("status", ctypes.c_int32),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("requests_done", ctypes.c_uint64), ("m_done", ctypes.c_uint64), ("prp_tests", ctypes.c_uint64),
        ("launches", ctypes.c_uint64), ("windows", ctypes.c_uint64), ("tables_built", ctypes.c_uint64),
        ("tables_evicted", ctypes.c_uint64), ("resident_bytes", ctypes.c_uint64), ("peak_bytes", ctypes.c_uint64),
        ("sieve_ms", ctypes.c_double), ("prp_ms", ctypes.c_double), ("busy_s", ctypes.c_double),
        ("preemptions", ctypes.c_uint64),
    ]


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python {PKG_DIR / 'build.py'}` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [s for s in EXPORTS if not hasattr(lib, s)]
    if missing:
        raise ImportError(f"{LIB_PATH} lacks {missing}")
    vp, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    P32, P64, PI32 = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32)
    lib.pg_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
    lib.pg_ctx_destroy.argtypes = [vp]
    lib.pg_ctx_stream.restype = vp
    lib.pg_ctx_stream.argtypes = [vp]
    lib.pg_measure_imad_peak.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    lib.pg_last_error.restype = ctypes.c_char_p
    lib.pg_version.restype = ctypes.c_char_p
    lib.pg_prp_batch.argtypes = [vp, P32, u32, u32, u32, PI32]
    lib.pg_prp_batch_device.argtypes = [vp, vp, u32, u32, u32, vp, vp]
    lib.pg_job_create.argtypes = [vp, ctypes.POINTER(JobParams), ctypes.POINTER(vp)]
    lib.pg_job_destroy.argtypes = [vp]
    lib.pg_job_get_info.argtypes = [vp, ctypes.POINTER(JobInfo)]
    lib.pg_job_k_words.argtypes = [vp, P32, P32]
    lib.pg_count_m.restype = u64
    lib.pg_count_m.argtypes = [u64, u64, u32]
    lib.pg_sieve_interval.argtypes = [vp, u64, u64, P64, P32]
    lib.pg_search.argtypes = [vp, u64, u64, i32, P64, P32, P32, ctypes.POINTER(SearchStats)]
    lib.pg_search_submit.argtypes = [vp, u64, u64, i32, u32, ctypes.POINTER(ctypes.c_uint64)]
    lib.pg_search_wait.argtypes = [vp, u64, P64, P32, P32, ctypes.POINTER(SearchStats)]
    lib.pg_job_stream.restype = vp
    lib.pg_job_stream.argtypes = [vp, i32]
    lib.pg_autotune.argtypes = [vp, ctypes.POINTER(JobParams), u64, u64, ctypes.POINTER(JobParams),
                                ctypes.POINTER(ctypes.c_double)]
    lib.pg_autotune_ex.argtypes = [vp, ctypes.POINTER(JobParams), u64, u64, u32, u32, ctypes.POINTER(TuneResult)]
    lib.pg_merit.restype = ctypes.c_double
    lib.pg_merit.argtypes = [ctypes.c_double, u64, u64]
    lib.pg_format_record.argtypes = [ctypes.c_char_p, ctypes.c_size_t, u64, ctypes.c_double, u64, u32, u32, u64]
    dbl = ctypes.c_double
    lib.pg_server_create.argtypes = [i32, ctypes.POINTER(ServerParams), ctypes.POINTER(vp)]
    lib.pg_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]
    lib.pg_server_wait.argtypes = [vp, u64, dbl, P64, P32, P32, ctypes.POINTER(RequestInfo)]
    lib.pg_server_next_done.argtypes = [vp, dbl, ctypes.POINTER(ctypes.c_uint64)]
    lib.pg_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    lib.pg_server_clock.restype = dbl
    lib.pg_server_clock.argtypes = [vp]
    lib.pg_server_destroy.argtypes = [vp]
    return lib


lib = _load()


def _check(rc: int) -> int:
    if rc < 0:
        raise PrimeGapError(rc, lib.pg_last_error().decode())
    return rc


def _p32(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _p64(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def version() -> str:
    return lib.pg_version().decode()


def count_m(m_start: int, m_inc: int, d: int) -> int:
    """m coprime to d in [m_start, m_start + m_inc) (count_num_m, gap_common.cpp:170-206)."""
    return int(lib.pg_count_m(m_start, m_inc, d))


def int_to_words(n: int, nwords: int) -> np.ndarray:
    return np.frombuffer(n.to_bytes(nwords * 4, "little"), dtype=np.uint32)


class Context:
    """A CUDA device and stream (the resources of test_runner_t's constructor)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib.pg_ctx_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream_ptr(self) -> int:
        """The context's cudaStream_t, e.g. for torch.cuda.ExternalStream."""
        return int(lib.pg_ctx_stream(self._h) or 0)

    def imad_peak(self) -> float:
        """Measured 32-bit integer multiply-adds per second of the whole device."""
        v = ctypes.c_double(0)
        _check(lib.pg_measure_imad_peak(self._h, ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            lib.pg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def prp_words(self, words: np.ndarray, rounds: int = 1) -> np.ndarray:
        """Bases passed per row of a (n, w) uint32 array of LE words."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        n, w = words.shape
        out = np.zeros(n, dtype=np.int32)
        _check(lib.pg_prp_batch(self._h, _p32(words), n, w, rounds,
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def prp(self, numbers, rounds: int = 1) -> np.ndarray:
        numbers = [int(x) for x in numbers]
        if not numbers:
            return np.zeros(0, dtype=np.int32)
        w = max(1, max((x.bit_length() + 31) // 32 for x in numbers))
        arr = np.stack([int_to_words(x, w) for x in numbers])
        return self.prp_words(arr, rounds)


class TestRunner:
    """Drop-in for test_runner_t<params> (miller_rabin.h:296-409).

    run_test(active, tests, results): tests are Python ints (the mpz_t
    batch), only the first `active` are computed, results[i] is set to
    (bases passed == rounds) for every i < len(tests) as the reference does
    (entries past `active` get 0 here instead of stale data).
    """
    __test__ = False  # not a pytest class

    def __init__(self, n: int, rounds: int = 1, device: int = 0, ctx: Context | None = None):
        self.n, self.rounds = n, rounds
        self.ctx = ctx or Context(device)

    def run_test(self, active: int, tests, results) -> None:
        if len(tests) == 0:
            return
        if len(tests) > self.n:
            raise ValueError(f"tests({len(tests)}) > n({self.n})")
        to_run = min(active, len(tests))
        for i in range(to_run):
            t = int(tests[i])
            if t <= 1 or t % 2 == 0:
                raise ValueError("candidates must be odd and > 1")
        passed = self.ctx.prp(list(tests[:to_run]), self.rounds) if to_run else []
        for i in range(len(tests)):
            results[i] = int(i < to_run and passed[i] == self.rounds)


@dataclasses.dataclass
class SearchResult:
    ms: np.ndarray
    prev_gap: np.ndarray
    next_gap: np.ndarray
    stats: dict


CONFIRM_ROUNDS = 16  # strong bases 2, 3, ..., 53 that both primes of a record pass


class Job:
    """K = P#/d, the sieve tables and the window buffers, resident on one device.

    confirm_merit: gaps with merit above it have both primes confirmed with
    confirm_rounds strong bases on the device before a search returns (the
    record double-check of overflow.cpp:164-177); 0 leaves that to records()."""

    def __init__(self, p: int, d: int, sl: int, max_prime: int, max_m_inc: int, max_m: int,
                 rounds: int = 1, small_limit: int = 0, ext_window: int = 0, flags: int = 0,
                 search_hits: int = 0, tpi: int = 0, ctx: Context | None = None, device: int = 0,
                 confirm_merit: float = 0.0, confirm_rounds: int = 0):
        self.ctx = ctx or Context(device)
        self.params = JobParams(p, d, sl, max_prime, max_m_inc, max_m, rounds, small_limit, ext_window, flags,
                                search_hits, tpi, confirm_merit, confirm_rounds, 0)
        self.confirm_merit = confirm_merit
        self.confirm_rounds = (confirm_rounds or CONFIRM_ROUNDS) if confirm_merit > 0 else 0
        h = ctypes.c_void_p()
        _check(lib.pg_job_create(self.ctx.handle, ctypes.byref(self.params), ctypes.byref(h)))
        self._h = h
        info = JobInfo()
        _check(lib.pg_job_get_info(self._h, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in info._fields_}
        self.p, self.d, self.sl, self.max_prime = p, d, sl, max_prime
        self.sly = sl // 2
        self.k_log = info.k_log
        nw = ctypes.c_uint32(0)
        _check(lib.pg_job_k_words(self._h, None, ctypes.byref(nw)))
        kw = np.zeros(nw.value, dtype=np.uint32)
        _check(lib.pg_job_k_words(self._h, _p32(kw), ctypes.byref(nw)))
        self.K = int.from_bytes(kw.tobytes(), "little")

    def close(self):
        if getattr(self, "_h", None):
            lib.pg_job_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def words_per_m(self) -> int:
        return self.info["words_per_m"]

    def sieve_interval(self, m_start: int, m_inc: int):
        """(ms, rows): rows[i] bit (Y + sl//2) set when ms[i]*K + 2Y has a factor <= max_prime."""
        n = count_m(m_start, m_inc, self.d)
        ms = np.zeros(n, dtype=np.uint64)
        rows = np.zeros((n, self.words_per_m), dtype=np.uint32)
        _check(lib.pg_sieve_interval(self._h, m_start, m_inc, _p64(ms), _p32(rows)))
        return ms, rows

    def search(self, m_start: int, m_inc: int, form: int = PG_SEARCH_PERSISTENT) -> SearchResult:
        n = count_m(m_start, m_inc, self.d)
        ms = np.zeros(n, dtype=np.uint64)
        prev = np.zeros(n, dtype=np.uint32)
        nxt = np.zeros(n, dtype=np.uint32)
        st = SearchStats()
        _check(lib.pg_search(self._h, m_start, m_inc, form, _p64(ms), _p32(prev), _p32(nxt), ctypes.byref(st)))
        return SearchResult(ms, prev, nxt, st.as_dict())

    def submit(self, m_start: int, m_inc: int, form: int = PG_SEARCH_PERSISTENT, flags: int = 0) -> int:
        """Enqueue the search of a window; returns a ticket for wait().  Up to
        PG_SEARCH_SLOTS windows may be in flight (they overlap on the device)."""
        t = ctypes.c_uint64(0)
        _check(lib.pg_search_submit(self._h, m_start, m_inc, form, flags, ctypes.byref(t)))
        if not hasattr(self, "_pending"):
            self._pending = {}
        self._pending[t.value] = count_m(m_start, m_inc, self.d)
        return t.value

    def wait(self, ticket: int) -> SearchResult:
        n = self._pending.pop(ticket)
        ms = np.zeros(n, dtype=np.uint64)
        prev = np.zeros(n, dtype=np.uint32)
        nxt = np.zeros(n, dtype=np.uint32)
        st = SearchStats()
        _check(lib.pg_search_wait(self._h, ticket, _p64(ms), _p32(prev), _p32(nxt), ctypes.byref(st)))
        return SearchResult(ms, prev, nxt, st.as_dict())

    def stream_ptr(self, slot: int) -> int:
        """cudaStream_t of a window slot (for CUDA-event timing)."""
        return int(lib.pg_job_stream(self._h, slot) or 0)

    def merits(self, res: SearchResult) -> np.ndarray:
        return np.array([merit(self.k_log, int(m), int(a) + int(b))
                         for m, a, b in zip(res.ms, res.prev_gap, res.next_gap)])

    def records(self, res: SearchResult, min_merit: float) -> list[str]:
        """Record lines of every gap with merit > min_merit (overflow.cpp:162-188, strict >).

        Every record is confirmed (overflow.cpp:164-177): the search already
        confirmed both primes of such gaps when the job's confirm_merit is at
        most min_merit; otherwise both primes are tested here with
        CONFIRM_ROUNDS strong bases on the device, and a prime that fails
        raises PrimeGapError (the gap would not be exact: search that window
        with confirm_merit <= min_merit, which searches on past such a
        prime)."""
        lines = records(res, self.k_log, self.p, self.d, min_merit)
        if lines and not (0 < self.confirm_merit <= min_merit and self.confirm_rounds >= CONFIRM_ROUNDS):
            ends = []
            for line in lines:
                f = line.split()
                m, prev, gap = int(f[2]), int(f[-1]), int(f[0])
                ends += [m * self.K - prev, m * self.K - prev + gap]
            passed = self.ctx.prp(ends, rounds=CONFIRM_ROUNDS)
            bad = [x for x, v in zip(ends, passed) if v != CONFIRM_ROUNDS]
            if bad:
                raise PrimeGapError(-6, f"{len(bad)} record prime(s) failed the {CONFIRM_ROUNDS}-base "
                                        "confirmation: search with confirm_merit <= min_merit")
        return lines


def records(res: SearchResult, k_log: float, p: int, d: int, min_merit: float) -> list[str]:
    """Record lines of every gap of res with merit > min_merit (overflow.cpp:162-188, strict >)."""
    gaps = res.prev_gap.astype(np.float64) + res.next_gap.astype(np.float64)
    approx = gaps / (k_log + np.log(np.maximum(res.ms.astype(np.float64), 1.0)))
    out = []
    # numpy's log may differ from libm's in the last ulp: pre-filter with a
    # margin, then decide with the exact formula of overflow.cpp:162
    for i in np.nonzero(approx > min_merit - 1e-6)[0]:
        m, pg, ng = int(res.ms[i]), int(res.prev_gap[i]), int(res.next_gap[i])
        mer = merit(k_log, m, pg + ng)
        if mer > min_merit:
            out.append(format_record(pg + ng, mer, m, p, d, pg))
    return out


@dataclasses.dataclass
class ServedResult(SearchResult):
    info: dict


class Server:
    """Continuous-batching gap search on one device (pg_server_*).

    submit() queues a request of any (p, d, sl, max_prime, m range) and
    returns its id at once; a worker thread in the library packs windows of
    all admitted requests that share an operand layout into common search
    launches.  wait(id) returns the request's gaps like Job.search."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, batch_m: int = 0, window_m: int = 0,
                 max_windows: int = 0, max_sl: int = 0, small_limit: int = 0, ext_window: int = 0, tpi: int = 0,
                 warps_per_sm: int = 0, slots: int = 0, preempt_us: int = 0):
        self.params = ServerParams(hbm_budget, batch_m, window_m, max_windows, max_sl, small_limit, ext_window,
                                   tpi, warps_per_sm, slots, preempt_us)
        h = ctypes.c_void_p()
        _check(lib.pg_server_create(device, ctypes.byref(self.params), ctypes.byref(h)))
        self._h = h
        self._d = {}

    def close(self):
        if getattr(self, "_h", None):
            lib.pg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, p: int, d: int, sl: int, max_prime: int, m_start: int, m_inc: int, rounds: int = 1) -> int:
        rq = Request(p, d, sl, rounds, max_prime, m_start, m_inc)
        i = ctypes.c_uint64(0)
        _check(lib.pg_server_submit(self._h, ctypes.byref(rq), ctypes.byref(i)))
        self._d[i.value] = (d, count_m(m_start, m_inc, d))
        return i.value

    def wait(self, rid: int, timeout: float = -1.0) -> ServedResult:
        """The request's gaps (ascending m) and its timing; raises PrimeGapError
        with PG_ERR_TIMEOUT (-5) if it is not done within timeout seconds."""
        _, n = self._d[rid]
        ms = np.zeros(n, dtype=np.uint64)
        prev = np.zeros(n, dtype=np.uint32)
        nxt = np.zeros(n, dtype=np.uint32)
        info = RequestInfo()
        rc = lib.pg_server_wait(self._h, rid, timeout, _p64(ms), _p32(prev), _p32(nxt), ctypes.byref(info))
        if rc != -5:
            self._d.pop(rid, None)
        _check(rc)
        return ServedResult(ms, prev, nxt, {}, {f: getattr(info, f) for f, _ in info._fields_})

    def next_done(self, timeout: float = -1.0) -> int | None:
        """Id of the oldest finished request not yet returned here, None on timeout."""
        i = ctypes.c_uint64(0)
        rc = lib.pg_server_next_done(self._h, timeout, ctypes.byref(i))
        if rc == -5:
            return None
        _check(rc)
        return i.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib.pg_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def clock(self) -> float:
        """Seconds since the server started (the clock of the request timings)."""
        return float(lib.pg_server_clock(self._h))


JOB_KNOBS = ("rounds", "small_limit", "ext_window", "flags", "search_hits", "tpi")


def autotune(p: int, d: int, sl: int, max_prime: int, m_start: int, m_inc: int, ctx: Context | None = None,
             cache: str | pathlib.Path | None = None, **knobs) -> tuple[dict, float]:
    """Times the sample window [m_start, m_start + m_inc) with candidate sieve
    tiles and operand layouts (pg_autotune) and returns (best knobs, ms per
    window).  With `cache`, results are kept in that JSON file, keyed by the
    job's shape and the operand bit length, and reused."""
    import json
    key = None
    if cache is not None:
        cache = pathlib.Path(cache)
        store = json.loads(cache.read_text()) if cache.exists() else {}
        key = f"P{p}/d{d}/sl{sl}/limit{max_prime}/minc{m_inc}/m{m_start.bit_length()}bits/" + \
              "/".join(f"{k}={knobs[k]}" for k in sorted(knobs))
        if key in store:
            return store[key]["knobs"], store[key]["ms"]
    ctx = ctx or Context(0)
    base = JobParams(p, d, sl, max_prime, m_inc, m_start + m_inc, knobs.get("rounds", 1), knobs.get("small_limit", 0),
                     knobs.get("ext_window", 0), knobs.get("flags", 0), knobs.get("search_hits", 0), knobs.get("tpi", 0),
                     0.0, 0, 0)
    best = JobParams()
    ms = ctypes.c_double(0)
    _check(lib.pg_autotune(ctx.handle, ctypes.byref(base), m_start, m_inc, ctypes.byref(best), ctypes.byref(ms)))
    out = {k: getattr(best, k) for k in JOB_KNOBS}
    if key is not None:
        store[key] = {"knobs": out, "ms": ms.value}
        cache.write_text(json.dumps(store, indent=1))
    return out, ms.value


def autotune_ex(p: int, d: int, sl: int, max_prime: int, m_start: int, m_inc: int, ctx: Context | None = None,
                windows: bool = False, reps: int = 0, cache: str | pathlib.Path | None = None,
                **knobs) -> dict:
    """pg_autotune_ex: threads per number, sieve tile bound, PRP warps per SM and (windows=True) the m per
    window, timed with PG_SEARCH_SLOTS windows of the sample [m_start, m_start + m_inc) in flight.  Returns
    {"knobs": job knobs, "warps_per_sm", "window_m", "m_per_sec", "first_m_per_sec", "settings"}.  With
    `cache`, results are kept in that JSON file keyed by the operand width, threads per number asked, sl and
    the sample, and reused."""
    import json
    key = None
    if cache is not None:
        cache = pathlib.Path(cache)
        store = json.loads(cache.read_text()) if cache.exists() else {}
        K = 1
        for q in range(2, p + 1):
            if all(q % r for r in range(2, int(q ** 0.5) + 1)):
                K *= q
        bits = (K // d * (m_start + m_inc)).bit_length()
        key = (f"bits{bits}/tpi{knobs.get('tpi', 0)}/sl{sl}/P{p}/d{d}/limit{max_prime}/m{m_start}+{m_inc}/"
               f"win{int(windows)}/" + "/".join(f"{k}={knobs[k]}" for k in sorted(knobs)))
        if key in store:
            return store[key]
    ctx = ctx or Context(0)
    base = JobParams(p, d, sl, max_prime, m_inc, m_start + m_inc, knobs.get("rounds", 1), knobs.get("small_limit", 0),
                     knobs.get("ext_window", 0), knobs.get("flags", 0), knobs.get("search_hits", 0),
                     knobs.get("tpi", 0), knobs.get("confirm_merit", 0.0), knobs.get("confirm_rounds", 0), 0)
    res = TuneResult()
    _check(lib.pg_autotune_ex(ctx.handle, ctypes.byref(base), m_start, m_inc, PG_TUNE_WINDOW if windows else 0,
                              reps, ctypes.byref(res)))
    out = {"knobs": {k: getattr(res.params, k) for k in JOB_KNOBS}, "warps_per_sm": res.warps_per_sm,
           "window_m": res.window_m, "m_per_sec": res.m_per_sec, "first_m_per_sec": res.first_m_per_sec,
           "settings": res.settings}
    if key is not None:
        store[key] = out
        cache.write_text(json.dumps(store, indent=1))
    return out


def merit(k_log: float, m: int, gap: int) -> float:
    """gap / (K_log + log(m)) (overflow.cpp:162)."""
    return lib.pg_merit(k_log, m, gap)


def format_record(gap: int, merit_value: float, m: int, p: int, d: int, prev_gap: int) -> str:
    """"{gap} {merit:.3f} {m} * {P}# / {D} - {prev_gap}" (overflow.cpp:180-182)."""
    buf = ctypes.create_string_buffer(256)
    n = _check(lib.pg_format_record(buf, 256, gap, merit_value, m, p, d, prev_gap))
    return buf.raw[:n].decode()


def k_log_of(K: int) -> float:
    """log(K) exactly as _log (gap_common.cpp:44-48): 53-bit truncated mantissa."""
    b = K.bit_length()
    top = K >> (b - 53) if b > 53 else K << (53 - b)
    return math.log(top / 2.0 ** 53) + math.log(2.0) * b
