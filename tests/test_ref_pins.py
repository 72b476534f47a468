"""Parity pinned to the reference's own code (tests/golden/ref_pins.json, made by
tests/golden/make_ref_golden.py from oracle/_ref/ref_tool -- the reference's
unmodified gap_common.cpp and overflow.cpp -- and the reference's
misc/misc_utils.py and misc/record_check.py).

CPU tests: the oracle and the library's host functions (count of coprime m,
K_log, merit, record format) against those values; the record lines the
reference's overflow thread printed against the oracle's GMP gaps run through
the library's merit and record formatting.  When the reference tree and the
built ref_tool are present (this container, not a GPU box), the tool is run
again and must reproduce the fixture.  The GPU side is tests/test_ref_pins_gpu.py.
"""
from __future__ import annotations

import ast
import hashlib
import pathlib
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

REF = pathlib.Path("/root/reference")
TOOL = ROOT / "oracle" / "_ref" / "ref_tool"


@pytest.fixture(scope="module")
def pins():
    return golden("ref_pins.json")


def reference_records(pg, run, k_log, ms, prev, nxt) -> list[str]:
    """The record lines overflow.cpp:145-188 prints for these gaps: only m whose
    next gap reaches MIN_GAP_TO_CONTINUE get a previous prime and a merit;
    merit > min_merit (strict) prints the line."""
    out = []
    for m, a, b in zip(ms, prev, nxt):
        m, a, b = int(m), int(a), int(b)
        if b < run["min_gap_to_continue"]:
            continue
        mer = pg.merit(k_log, m, a + b)
        if mer > run["min_merit"]:
            out.append(pg.format_record(a + b, mer, m, run["P"], run["d"], a))
    return out


@pytest.mark.parametrize("key", ["337/2310", "503/2190", "907/210", "3001/2190", "151/2310", "257/210",
                                 "701/30", "1009/2310"])
def test_k_and_k_log_equal_the_reference(pg, oracle, pins, key):
    """init_K and calc_log_K of gap_common.cpp, bit for bit: the oracle's K and K_log, and the library's
    K_log formula (pg.k_log_of mirrors the host bignum's big_log)."""
    P, d = map(int, key.split("/"))
    ref = pins["k"][key]
    with oracle.Job(P, d, 100, 10_000, threads=1) as j:
        assert j.K == int(ref["hex"], 16) and j.K.bit_length() == ref["bits"]
        assert j.K_log == ref["k_log"]
    assert pg.k_log_of(int(ref["hex"], 16)) == ref["k_log"]


def test_count_num_m_equals_the_reference(pg, oracle, pins):
    for w in pins["count_num_m"]:
        assert pg.count_m(w["m_start"], w["m_inc"], w["d"]) == w["count"], w
        assert len(oracle.coprime_ms(w["m_start"], w["m_inc"], w["d"])) == w["count"], w


def test_coprime_m_lists_equal_calc_valid_mi(oracle, pins):
    """The coprime m of each window, as offsets from m_start, hash like misc_utils.calc_valid_mi's."""
    for w in pins["valid_mi"]:
        ms = oracle.coprime_ms(w["m_start"], w["m_inc"], w["d"]).astype(np.int64) - w["m_start"]
        assert len(ms) == w["count"]
        assert hashlib.sha256(ms.tobytes()).hexdigest() == w["sha256"], w


def test_primes_below_a_million_equal_get_sieve_primes(oracle, pins):
    ps = oracle.primes(2, 1_000_000)
    if ps[0] == 3:  # the oracle's generator lists the odd primes; get_sieve_primes starts at 2
        ps = np.concatenate([np.array([2], dtype=ps.dtype), ps])
    ref = pins["primes_1e6"]
    assert len(ps) == ref["count"] and int(ps.sum()) == ref["sum"] and int(ps[-1]) == ref["last"]


@pytest.mark.parametrize("run_idx", [0, 1, 2])
def test_reference_record_lines_from_oracle_gaps(pg, oracle, pins, run_idx):
    """The record lines the reference's overflow thread printed (its GMP gaps, merit, double-check and
    std::format line) equal the oracle's GMP gaps run through pg_merit and pg_format_record."""
    run = pins["records"][run_idx]
    P, d = run["P"], run["d"]
    ms = oracle.coprime_ms(run["m_start"], run["span"], d)
    assert len(ms) == run["m_count"]
    if run_idx > 0:  # wider operands: the oracle's GMP on a prefix; the fixture cut to the same m
        ms = ms[:400]
    with oracle.Job(P, d, 100, 10_000) as oj:
        prev, nxt = oj.gmp_gaps(ms)
    k_log = pins["k"][f"{P}/{d}"]["k_log"]
    want = [ln for ln in run["lines"] if int(ln.split()[2]) <= int(ms[-1])]
    assert len(want) > 20
    assert reference_records(pg, run, k_log, ms, prev, nxt) == want


@pytest.mark.skipif(not (REF / "misc" / "record_check.py").exists(), reason="reference tree not mounted")
def test_record_lines_parse_with_the_reference_regex(pg, pins):
    """misc/record_check.py's record_format (read from its source: the module needs gmpy2) parses every
    line pg_format_record makes, into the same fields."""
    tree = ast.parse((REF / "misc" / "record_check.py").read_text())
    rx = None
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "record_format" for t in node.targets):
            rx = re.compile(*[ast.literal_eval(a) for a in node.value.args])
    assert rx is not None
    for run in pins["records"]:
        for ln in run["lines"][:50]:
            f = ln.split()
            gap, m, prev = int(f[0]), int(f[2]), int(f[-1])
            mine = pg.format_record(gap, float(f[1]), m, run["P"], run["d"], prev)
            g = rx.match(mine)
            assert g and g.group(0) == mine
            assert (int(g.group(1)), int(g.group(3)), g.group(5)) == (gap, m, f"{run['P']}#")
            assert int(g.group(7).replace("-", "").strip()) == prev


@pytest.mark.skipif(not (TOOL.exists() and REF.exists()), reason="oracle/_ref/ref_tool not built here")
def test_ref_tool_reproduces_the_fixture(pins, tmp_path):
    """The committed pins come from the reference code as built by oracle/Makefile (target ref)."""
    def tool(*args):
        return subprocess.run([str(TOOL), *map(str, args)], capture_output=True, text=True, check=True,
                              cwd=tmp_path).stdout
    for key in ("337/2310", "3001/2190"):
        f = dict(line.split(" ", 1) for line in tool("k", *key.split("/")).splitlines())
        assert int(f["hex"], 16) == int(pins["k"][key]["hex"], 16)
        assert float.fromhex(f["k_log"]) == pins["k"][key]["k_log"]
    for w in pins["count_num_m"][:6]:
        assert int(tool("count", w["m_start"], w["m_inc"], w["d"])) == w["count"]
    run = pins["records"][0]
    ms = [m for m in range(run["m_start"], run["m_start"] + 1500) if np.gcd(m, run["d"]) == 1]
    lines = [ln for ln in tool("overflow", run["P"], run["d"], run["m_inc"], run["min_merit"], *ms).splitlines()
             if re.match(r"^\d+ \d+\.\d{3} \d+ \* \d+# / \d+ - \d+$", ln)]
    assert lines == [ln for ln in run["lines"] if int(ln.split()[2]) < run["m_start"] + 1500]
