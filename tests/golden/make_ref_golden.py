"""Generates tests/golden/ref_pins.json from the reference's own code.

    make -C oracle ref && python tests/golden/make_ref_golden.py

Everything in the fixture comes from reference code run in this container
(the reference tree at /root/reference, read-only):

* oracle/_ref/ref_tool, the reference's unmodified gap_common.cpp and
  overflow.cpp compiled against the GMP 6.3.0 runtime (oracle/Makefile, target
  ref): K = P#/d and K_log (init_K / calc_log_K, gap_common.cpp:51-65),
  count_num_m (gap_common.cpp:170-206), get_sieve_primes (gap_common.cpp:
  256-278), and the record lines run_cpu_overflow_thread prints for a list of
  m (overflow.cpp:145-188: GMP next / prev prime, merit, the record
  double-check, the record format);
* misc/misc_utils.py, imported from the reference tree: count_num_m and
  calc_valid_mi (the coprime m offsets);
* misc/record_check.py's record regex (record_check.py:272-275), read from
  the source with ast (the module imports gmpy2 and primegapverify, absent
  here), applied to every record line.

The reference prints a record only when the next gap reaches
MIN_GAP_TO_CONTINUE (overflow.cpp:83-84, 154); the fixture stores that
threshold, computed with the reference's float arithmetic, beside each run.
"""
from __future__ import annotations

import ast
import hashlib
import importlib.util
import json
import math
import pathlib
import re
import subprocess
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
REF = pathlib.Path("/root/reference")
TOOL = ROOT / "oracle" / "_ref" / "ref_tool"
OUT = ROOT / "tests" / "golden" / "ref_pins.json"

CONFIGS = [  # (P, d, m_start, m_inc): the workloads' windows
    (337, 2310, 10_000_000, 10_000),
    (503, 2190, 1_000_000, 200_000),
    (907, 210, 1_000_000, 50_000),
    (3001, 2190, 1, 100_000),
]
EXTRA_K = [(151, 2310), (257, 210), (701, 30), (1009, 2310)]
# record runs: (P, d, m_inc passed to the reference, min_merit, (m_start, span))
RECORD_RUNS = [
    (337, 2310, 10_000, 1.0, (10_000_000, 10_000)),   # every m of the P=337 window
    (503, 2190, 200_000, 1.0, (1_000_000, 12_000)),   # the first 12 000 m of the P=503 window
    (907, 210, 50_000, 1.0, (1_000_000, 1_500)),      # the first 1 500 m of the P=907 window
]


def tool(*args, cwd=None) -> str:
    return subprocess.run([str(TOOL), *map(str, args)], capture_output=True, text=True, check=True,
                          cwd=cwd).stdout


def load_misc_utils():
    spec = importlib.util.spec_from_file_location("ref_misc_utils", REF / "misc" / "misc_utils.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def record_regex() -> re.Pattern:
    """The record_format regex of misc/record_check.py, evaluated from its source text."""
    tree = ast.parse((REF / "misc" / "record_check.py").read_text())
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "record_format" for t in node.targets):
            call = node.value
            assert isinstance(call, ast.Call) and call.func.attr == "compile"
            return re.compile(*[ast.literal_eval(a) for a in call.args])
    raise RuntimeError("record_format not found")


def min_gap_to_continue(k_log: float, m_inc: int, min_merit: float) -> float:
    """MIN_GAP_TO_CONTINUE of overflow.cpp:83-84 with its float / double steps."""
    mm = float(np.float32(min_merit))
    cont = np.float32(2.6 + math.log2(mm * math.log(2) + 1))
    return float(np.float32(float(cont) * (k_log + math.log(m_inc))))


def coprime(m_start: int, m_inc: int, d: int) -> list[int]:
    return [m for m in range(m_start, m_start + m_inc) if math.gcd(m, d) == 1]


def main() -> None:
    mu = load_misc_utils()
    rx = record_regex()
    out = {"source": "reference code run here: oracle/_ref/ref_tool (gap_common.cpp, overflow.cpp), "
                     "misc/misc_utils.py, misc/record_check.py's regex",
           "k": {}, "count_num_m": [], "valid_mi": [], "primes_1e6": None, "records": []}
    for P, d in [(c[0], c[1]) for c in CONFIGS] + EXTRA_K:
        f = dict(line.split(" ", 1) for line in tool("k", P, d).splitlines())
        out["k"][f"{P}/{d}"] = {"bits": int(f["bits"]), "hex": f["hex"], "k_log": float.fromhex(f["k_log"])}
    rng = np.random.default_rng(11)
    windows = [(c[2], c[3], c[1]) for c in CONFIGS] + [
        (int(rng.integers(1, 10**12)), int(rng.integers(1, 300_000)), int(d))
        for d in rng.choice([30, 210, 2190, 2310, 30030, 510510], 12)]
    for ms, mi, d in windows:
        c_ref = int(tool("count", ms, mi, d))
        c_py = mu.count_num_m(ms, mi, d)
        assert c_ref == c_py, (ms, mi, d)
        out["count_num_m"].append({"m_start": ms, "m_inc": mi, "d": d, "count": c_ref})
    for ms, mi, d in windows[:7]:
        vm = np.asarray(mu.calc_valid_mi(ms, mi, d), dtype=np.int64)
        out["valid_mi"].append({"m_start": ms, "m_inc": mi, "d": d, "count": int(len(vm)),
                                "sha256": hashlib.sha256(vm.tobytes()).hexdigest()})
    f = tool("primes", 1_000_000).split()
    out["primes_1e6"] = {"count": int(f[1]), "sum": int(f[3]), "last": int(f[5])}
    for P, d, m_inc, min_merit, (m0, span) in RECORD_RUNS:
        ms = coprime(m0, span, d)
        with tempfile.TemporaryDirectory() as tmp:
            text = tool("overflow", P, d, m_inc, min_merit, *ms, cwd=tmp)
            kept = (pathlib.Path(tmp) / f"records_{P}.txt").read_text().splitlines()
        lines = [ln for ln in text.splitlines() if rx.match(ln)]
        assert lines == kept, "stdout and records file disagree"
        k_log = out["k"][f"{P}/{d}"]["k_log"]
        out["records"].append({"P": P, "d": d, "m_inc": m_inc, "min_merit": min_merit, "m_start": m0, "span": span,
                               "m_count": len(ms), "min_gap_to_continue": min_gap_to_continue(k_log, m_inc, min_merit),
                               "lines": lines})
        print(f"P={P}: {len(lines)} record lines from {len(ms)} m")
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
