"""The oracle (CPU restatement of the reference path) against the golden fixtures."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden


def test_prp_vectors(oracle, prp_vectors):
    kinds = set()
    for it in prp_vectors["items"]:
        n = int(it["n"], 16)
        assert oracle.prp(n, 1) == it["sprp2"], it
        assert oracle.prp(n, 4) == it["mr4"], it
        kinds.add(it["kind"])
    assert {"prime", "composite", "spsp2", "carmichael"} <= kinds
    spsp = [int(it["n"], 16) for it in prp_vectors["items"] if it["kind"] == "spsp2"]
    assert any(n.bit_length() > 64 for n in spsp), "need multi-word strong pseudoprimes"
    # every strong base-2 pseudoprime passes base 2 and is composite for GMP
    for it in prp_vectors["items"]:
        if it["kind"] == "spsp2":
            assert it["sprp2"] == 1 and it["gmp"] == 0


def test_sieve_rows_golden(oracle):
    g = golden("sieve_rows.json")
    with oracle.Job(g["P"], g["d"], g["sl"], g["max_prime"]) as j:
        ms = oracle.coprime_ms(g["m_start"], g["m_inc"], g["d"])
        assert [int(m) for m in ms] == g["ms"]
        rows = j.sieve_m(ms)
        assert [hashlib.sha256(r.tobytes()).hexdigest() for r in rows] == g["row_sha256"]
        for m, row in g["full_rows"].items():
            i = g["ms"].index(int(m))
            assert [int(w) for w in rows[i]] == row


def test_sieve_per_x_equals_per_m(oracle):
    # the reference's loop order (one X row across all m) and the per-m form agree
    with oracle.Job(503, 2190, 2000, 3_000_000) as j:
        rows_x = j.sieve_x(1_000_000, 3_000)
        ms = oracle.coprime_ms(1_000_000, 3_000, 2190)
        assert np.array_equal(rows_x, j.sieve_m(ms))


def test_gaps_P337_golden(oracle):
    g = golden("gaps_P337_d2310.json")
    ms = np.array(g["ms"], dtype=np.uint64)
    assert len(ms) == 2079
    with oracle.Job(g["P"], g["d"], g["sl"], 1_000_000) as j:
        assert j.K_log == g["k_log"]
        # ground truth straight from GMP for the whole window
        prev, nxt = j.gmp_gaps(ms)
        assert list(prev) == g["prev_gap"] and list(nxt) == g["next_gap"]
        # the sieve + outward PRP search on a slice
        sl = slice(0, 120)
        p2, n2, _, tests = j.search(ms[sl], 1)
        assert list(p2) == g["prev_gap"][sl] and list(n2) == g["next_gap"][sl]
        assert tests > 0


def test_records_P337(oracle):
    import math
    g = golden("gaps_P337_d2310.json")
    recs = []
    for m, a, b in zip(g["ms"], g["prev_gap"], g["next_gap"]):
        mer = (a + b) / (g["k_log"] + math.log(m))
        if mer > g["min_merit"]:
            recs.append(f"{a + b} {mer:.3f} {m} * {g['P']}# / {g['d']} - {a}")
    assert recs == g["records"] and len(recs) > 0


@pytest.mark.parametrize("name", ["gaps_P503_d2190.json", "gaps_P907_d210.json"])
def test_gaps_samples_golden(oracle, name):
    g = golden(name)
    ms = np.array(g["ms"][:4], dtype=np.uint64)
    with oracle.Job(g["P"], g["d"], g["sl"], 1_000_000) as j:
        prev, nxt = j.gmp_gaps(ms)
        assert list(prev) == g["prev_gap"][:4] and list(nxt) == g["next_gap"][:4]
        p2, n2, _, _ = j.search(ms, 1)
        assert list(p2) == g["prev_gap"][:4] and list(n2) == g["next_gap"][:4]


def test_search_past_sl_uses_gmp_finishing(oracle):
    # SL far below the prime gaps: every side finishes with nextprime/prevprime
    ms = oracle.coprime_ms(10_000_000, 60, 2310)
    with oracle.Job(337, 2310, 20, 100_000) as j:
        prev, nxt, ovf, _ = j.search(ms, 1)
        gp, gn = j.gmp_gaps(ms)
        assert np.array_equal(prev, gp) and np.array_equal(nxt, gn)
        assert ovf.any()
