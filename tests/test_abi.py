"""The C-ABI library loads and exports every declared symbol; host-only helpers
(no GPU needed) agree with the oracle and the reference's formulas."""
from __future__ import annotations

import math
import re
import subprocess
import sys

import pytest

from conftest import ROOT


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "primegap.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    fns = declared_functions()
    for f in ("pg_ctx_create", "pg_prp_batch", "pg_job_create", "pg_sieve_interval", "pg_search"):
        assert f in fns


def test_library_exports_every_declared_symbol(pg):
    out = subprocess.run(["nm", "-D", "--defined-only", str(pg.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (pg_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    assert set(declared_functions()) <= set(pg.EXPORTS)


@pytest.mark.parametrize("m_start,m_inc,d", [(10_000_000, 10_000, 2310), (1_000_000, 200_000, 2190),
                                             (1, 100_000, 2190), (999_999, 12_345, 210), (7, 1, 30)])
def test_count_m_matches_oracle(pg, oracle, m_start, m_inc, d):
    assert pg.count_m(m_start, m_inc, d) == len(oracle.coprime_ms(m_start, m_inc, d))


def test_counts_of_the_benchmark_windows(pg):
    # coprime m of the four benchmark windows: 2,079 / 52,604 / 11,429 / 26,300
    assert pg.count_m(10_000_000, 10_000, 2310) == 2079
    assert pg.count_m(1_000_000, 200_000, 2190) == 52604
    assert pg.count_m(1_000_000, 50_000, 210) == 11429
    assert pg.count_m(1, 100_000, 2190) == 26300


@pytest.mark.parametrize("P,d", [(337, 2310), (503, 2190), (907, 210), (3001, 2190), (151, 2310)])
def test_k_log_matches_gmp(pg, oracle, P, d):
    with oracle.Job(P, d, 100, 10_000, threads=1) as j:
        assert pg.k_log_of(j.K) == j.K_log


def test_merit_formula(pg):
    k_log = 303.87395620173214
    for m, gap in [(10_000_003, 692), (1_000_001, 15000), (1, 2)]:
        assert pg.merit(k_log, m, gap) == gap / (k_log + math.log(m))


def test_record_format(pg):
    line = pg.format_record(15234, 22.51849, 1000003, 503, 2190, 7342)
    assert line == "15234 22.518 1000003 * 503# / 2190 - 7342"
    # parses with the record regex of misc/record_check.py:430-434
    assert re.match(r"(\d+)\s+(\d+\.\d+)\s+(\d+)\s*\*\s*(\d+)#\s*/\s*(\d+)\s*-\s*(\d+)", line)


def test_context_without_gpu_reports_an_error(pg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pg.PrimeGapError):
        pg.Context(0)


def test_server_without_gpu_reports_an_error(pg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pg.PrimeGapError):
        pg.Server(0)
    import ctypes
    rq = pg.Request(337, 2310, 1000, 1, 10**6, 10**7, 100)
    i = ctypes.c_uint64(0)
    assert pg.lib.pg_server_submit(None, ctypes.byref(rq), ctypes.byref(i)) == -1
    assert pg.lib.pg_server_destroy(None) == 0


def test_records_keep_strictly_greater_merits(pg):
    """records(): merit > min_merit strictly (overflow.cpp:164), exact formula after the numpy pre-filter."""
    import numpy as np
    k_log = 303.87395620173214
    ms = np.array([10_000_003, 10_000_019, 10_000_031], dtype=np.uint64)
    prev = np.array([300, 1000, 20], dtype=np.uint32)
    nxt = np.array([392, 1200, 10], dtype=np.uint32)
    res = pg.SearchResult(ms, prev, nxt, {})
    m1 = pg.merit(k_log, 10_000_003, 692)
    assert pg.records(res, k_log, 337, 2310, m1) == [pg.format_record(2200, pg.merit(k_log, 10_000_019, 2200),
                                                                      10_000_019, 337, 2310, 1000)]
    assert len(pg.records(res, k_log, 337, 2310, m1 - 1e-9)) == 2
    assert pg.records(res, k_log, 337, 2310, 100.0) == []


def test_format_record_rejects_a_short_buffer(pg):
    import ctypes
    buf = ctypes.create_string_buffer(8)
    rc = pg.lib.pg_format_record(buf, 8, 15234, 22.5, 1000003, 503, 2190, 7342)
    assert rc == -1 and "too small" in pg.lib.pg_last_error().decode()


def test_package_without_its_library_refuses_to_import(tmp_path):
    """No CPU fallback: a package copy whose libprimegap.so is absent raises on import."""
    import shutil
    pkg = tmp_path / "pkg"
    shutil.copytree(ROOT / "prime-gap-gpu_b200", pkg, ignore=shutil.ignore_patterns("build", "__pycache__"))
    code = ("import importlib.util, sys\n"
            f"spec = importlib.util.spec_from_file_location('pgcopy', r'{pkg / '__init__.py'}', "
            f"submodule_search_locations=[r'{pkg}'])\n"
            "m = importlib.util.module_from_spec(spec)\n"
            "sys.modules['pgcopy'] = m\n"
            "spec.loader.exec_module(m)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode != 0
    assert "ImportError" in r.stderr and "libprimegap.so is missing" in r.stderr


def test_struct_layouts_match_the_header(pg, tmp_path):
    """Every ctypes mirror of a header struct has the C sizes and field offsets (gcc on the header)."""
    import ctypes
    mirrors = {"pg_job_params": pg.JobParams, "pg_job_info": pg.JobInfo, "pg_search_stats": pg.SearchStats,
               "pg_server_params": pg.ServerParams, "pg_request": pg.Request, "pg_request_info": pg.RequestInfo,
               "pg_server_stats": pg.ServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "primegap.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for cname, cls in mirrors.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, f"{cname}.{f}"
