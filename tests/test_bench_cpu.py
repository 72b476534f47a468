"""bench.py's reference arm (CPU only): one JSON line in the contract's shape,
and the ranks other than 0 of a multi-rank launch print nothing."""
from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(env_extra: dict) -> subprocess.CompletedProcess:
    env = {**os.environ, **env_extra}
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], capture_output=True, text=True, env=env, cwd=ROOT, timeout=600)


def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "m/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["metric"].startswith("m/sec searched")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "m/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "P=503 d=2190" in d["config"]["workload"]


def test_reference_arm_other_ranks_stay_silent():
    r = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_roofline_work_per_test():
    """The limb-product counts behind the bench line's roofline: the fixed formula 2*L^2*(B + ceil(B/5))
    and the kernel's own work per strong base-2 test (B - 1 squarings of L(L+1)/2 + L^2 + L products)."""
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.products_per_test(703) == 816_992          # P=503: 703-bit N, 22 words
    assert bench.products_per_test(462) == 249_750          # P=337
    assert bench.products_per_test(1264) == 4_854_400       # P=907
    assert bench.kernel_products_per_test(703, 22) == 532_818
    assert bench.kernel_products_per_test(703, 22) / bench.products_per_test(703) < 0.66
