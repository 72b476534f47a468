"""Builds libprimegap.so (CUDA kernels + C ABI) in-tree for sm_100a.

    python prime-gap-gpu_b200/build.py [--force] [--jobs N]

Objects go to prime-gap-gpu_b200/build/; the PRP kernels are compiled once
per limb count listed in csrc/pg_limbs.h, in parallel.  ptxas register and
spill reports are kept next to the objects (build/*.ptxas.txt).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import re
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "build"
LIB = BUILD / "libprimegap.so"
CLI = BUILD / "gap_search_gpu"
ROOT = PKG.parent

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
              f"-I{ROOT / 'include'}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def limbs_header() -> str:
    """pg_limbs.h with its continued lines joined."""
    return (CSRC / "pg_limbs.h").read_text().replace("\\\n", " ")


def limb_list() -> list[int]:
    m = re.search(r"#define PG_LIMB_LIST\(X\)(.*)", limbs_header())
    return [int(v) for v in re.findall(r"X\((\d+)\)", m.group(1))]


def group_list() -> list[tuple[int, int]]:
    m = re.search(r"#define PG_GROUP_LIST\(X\)(.*)", limbs_header())
    return [(int(a), int(b)) for a, b in re.findall(r"X\((\d+),\s*(\d+)\)", m.group(1))]


def headers() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "primegap.h"]


def units() -> list[tuple[pathlib.Path, pathlib.Path, list[str]]]:
    out = []
    for name in ("pg_kernels", "pg_dispatch", "pg_api", "pg_server", "pg_noalloc"):
        src = CSRC / f"{name}.cu"
        if src.exists():
            out.append((src, BUILD / f"{name}.o", []))
    for L in limb_list():
        out.append((CSRC / "pg_inst.cu", BUILD / f"pg_inst_{L}.o", [f"-DPG_LIMBS={L}"]))
    for T, LT in group_list():
        out.append((CSRC / "pg_ginst.cu", BUILD / f"pg_ginst_{T}x{LT}.o", [f"-DPG_GT={T}", f"-DPG_GLT={LT}"]))
    return out


def stale(obj: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def compile_one(src: pathlib.Path, obj: pathlib.Path, extra: list[str]) -> str:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    obj.with_suffix(".ptxas.txt").write_text(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name} {' '.join(extra)}:\n{r.stderr[-4000:]}")
    return obj.name


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    deps = headers()
    todo = [(s, o, e) for s, o, e in units() if force or stale(o, deps + [s])]
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(jobs) as ex:
            for name in ex.map(lambda u: compile_one(*u), todo):
                if verbose:
                    print("built", name, flush=True)
    objs = [o for _, o, _ in units()]
    if force or todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        if verbose:
            print("linked", LIB, flush=True)
    cli_src = CSRC / "gap_search_gpu.cpp"
    if cli_src.exists() and (force or not CLI.exists() or CLI.stat().st_mtime < max(
            LIB.stat().st_mtime, cli_src.stat().st_mtime)):
        cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", f"-I{ROOT / 'include'}", str(cli_src),
               "-o", str(CLI), f"-L{BUILD}", "-lprimegap", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stderr[-4000:]}")
        if verbose:
            print("built", CLI, flush=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    build(a.force, a.jobs, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
