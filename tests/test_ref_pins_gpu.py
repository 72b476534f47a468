"""The CUDA search against values the reference's own code produced
(tests/golden/ref_pins.json: the reference's gap_common.cpp and overflow.cpp
built into oracle/_ref/ref_tool, and its misc/misc_utils.py).

* K and K_log of every workload's job equal init_K / calc_log_K.
* The coprime m of a window hash like misc_utils.calc_valid_mi's.
* The record lines: the reference's overflow thread ran GMP next/prev prime
  from m*K for every m of a window and printed the records it found
  (overflow.cpp:145-188); the GPU search of the same window, with record
  confirmation on, gives exactly those lines once the same MIN_GAP_TO_CONTINUE
  filter is applied (the GPU search reports every gap; the reference skips
  the previous prime of m whose next gap is short, overflow.cpp:154).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden
from test_ref_pins import reference_records

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pins():
    return golden("ref_pins.json")


@pytest.mark.parametrize("P,d", [(337, 2310), (503, 2190), (907, 210), (3001, 2190)])
def test_job_k_equals_init_k(pg, pins, P, d):
    ref = pins["k"][f"{P}/{d}"]
    with pg.Job(P, d, 1_000, 1_000_000, max_m_inc=100, max_m=100_000) as job:
        assert job.K == int(ref["hex"], 16)
        assert job.info["k_bits"] == ref["bits"]
        assert job.k_log == ref["k_log"]


@pytest.mark.parametrize("run_idx,sl,limit", [(0, 7_500, 100_000_000), (1, 10_000, 2_000_000_000),
                                              (2, 18_000, 10_000_000_000)])
def test_gpu_records_equal_the_reference_overflow_thread(pg, pins, run_idx, sl, limit):
    run = pins["records"][run_idx]
    P, d = run["P"], run["d"]
    with pg.Job(P, d, sl, limit, max_m_inc=run["span"], max_m=run["m_start"] + run["span"],
                confirm_merit=run["min_merit"]) as job:
        res = job.search(run["m_start"], run["span"])
        assert len(res.ms) == run["m_count"]
        got = reference_records(pg, run, job.k_log, res.ms, res.prev_gap, res.next_gap)
        assert res.stats["confirm_tests"] > 0
    assert got == run["lines"]
    assert len(got) > 50


def test_gpu_coprime_m_equal_calc_valid_mi(pg, pins):
    w = pins["valid_mi"][0]  # the P=337 window
    assert (w["m_start"], w["m_inc"], w["d"]) == (10_000_000, 10_000, 2310)
    with pg.Job(337, 2310, 600, 1_000_000, max_m_inc=w["m_inc"], max_m=w["m_start"] + w["m_inc"]) as job:
        ms, _ = job.sieve_interval(w["m_start"], w["m_inc"])
    off = ms.astype(np.int64) - w["m_start"]
    assert len(off) == w["count"] and hashlib.sha256(off.tobytes()).hexdigest() == w["sha256"]
