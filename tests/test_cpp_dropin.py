"""The C++ drop-in header (include/primegap_runner.hpp) compiles against the
reference's call shape, links libprimegap.so, and (on a GPU) gives the
reference's results."""
from __future__ import annotations

import subprocess

import pytest

from conftest import ROOT

GMP_SO = "/lib/x86_64-linux-gnu/libgmp.so.10"


def build_dropin(pg, tmp_path):
    exe = tmp_path / "runner_dropin"
    lib_dir = pg.LIB_PATH.parent
    cmd = ["g++", "-O1", "-std=c++17", "-Wall", f"-I{ROOT / 'include'}", f"-I{ROOT / 'tests' / 'cpp' / 'shim'}",
           str(ROOT / "tests" / "cpp" / "runner_dropin.cpp"), "-o", str(exe), f"-L{lib_dir}", "-lprimegap",
           GMP_SO, f"-Wl,-rpath,{lib_dir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dropin_compiles_and_links(pg, tmp_path):
    assert build_dropin(pg, tmp_path).exists()


def test_cli_help(pg):
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    out = subprocess.run([str(cli), "-h"], capture_output=True, text=True)
    assert out.returncode == 0
    for flag in ("-p", "-d", "--mstart", "--minc", "--min-merit", "--max-prime", "--cpu-fraction", "--sl"):
        assert flag in out.stdout


@pytest.mark.gpu
def test_dropin_results(pg, tmp_path):
    exe = build_dropin(pg, tmp_path)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    res = dict(zip(map(int, out[0::2]), map(int, out[1::2])))
    # 2^521-1 prime, 2^521+1 composite, 2047 passes base 2, 101 prime, 2^127-1 prime, past `active`: 0
    assert res == {0: 1, 1: 0, 2: 1, 3: 1, 4: 1, 5: 0}


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["--chunk", "1500"], ["--chunk", "1500", "--warps-per-sm", "0"],
                                   ["--chunk", "2500", "--form", "plain"]])
def test_cli_records(pg, tmp_path, extra):
    """gap_search_gpu on the P=337 window prints the GMP records of merit > 5, in m order, also when the
    range is cut into chunks that run two at a time."""
    from conftest import golden
    g = golden("gaps_P337_d2310.json")
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    out = subprocess.run([str(cli), "-p", "337", "-d", "2310", "--mstart", "10000000", "--minc", "10000",
                          "--max-prime", "100", "--min-merit", "5", "--sl", "7500", "--ranges", "1", "-q", *extra],
                         capture_output=True, text=True, cwd=tmp_path, check=True).stdout
    import re
    rec = re.compile(r"^\d+ \d+\.\d{3} \d+ \* \d+# / \d+ - \d+$")
    lines = [line for line in out.splitlines() if rec.match(line)]
    assert lines == g["records"]
    assert (tmp_path / "records_337.txt").read_text().splitlines() == g["records"]


@pytest.mark.gpu
def test_cli_confirms_records_and_spot_checks(pg, tmp_path):
    """The stats block: every record's primes were confirmed on the device (15 extra bases x 2 sides per
    record, none past them) and GMP spot-checked found primes; the records are still GMP's."""
    from conftest import golden
    g = golden("gaps_P337_d2310.json")
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    out = subprocess.run([str(cli), "-p", "337", "-d", "2310", "--mstart", "10000000", "--minc", "10000",
                          "--max-prime", "100", "--min-merit", "5", "--sl", "7500", "--ranges", "1",
                          "--spot-check", "3"], capture_output=True, text=True, cwd=tmp_path, check=True).stdout
    import re
    rec = re.compile(r"^\d+ \d+\.\d{3} \d+ \* \d+# / \d+ - \d+$")
    assert [line for line in out.splitlines() if rec.match(line)] == g["records"]
    confirm = int(re.search(r"confirm tests\s*: (\d+)", out).group(1))
    merits = [pg.merit(g["k_log"], m, a + b) for m, a, b in zip(g["ms"], g["prev_gap"], g["next_gap"])]
    assert confirm == 15 * 2 * sum(x > 5 - 1e-6 for x in merits) and confirm > 0
    spot = int(re.search(r"spot checked\s*: (\d+)", out).group(1))
    assert spot == 6  # three m, both primes, one window


def test_cli_resume_file_checks(pg, tmp_path):
    """A progress file of another search is refused; a finished one ends the run at once (no device use)."""
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    prog = tmp_path / "progress.txt"
    prog.write_text("337 2310 5000 10005000 1\n")
    r = subprocess.run([str(cli), "-p", "337", "-d", "210", "--mstart", "10000000", "--minc", "5000",
                        "--max-prime", "100", "--ranges", "2", "--resume", str(prog), "-q"],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "does not hold the progress" in r.stderr
    r = subprocess.run([str(cli), "-p", "337", "-d", "2310", "--mstart", "10000000", "--minc", "5000",
                        "--max-prime", "100", "--ranges", "1", "--resume", str(prog), "-q"],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and prog.read_text() == "337 2310 5000 10005000 1\n"


@pytest.mark.gpu
def test_cli_resume_continues(pg, tmp_path):
    """Two runs with a progress file search the P=337 window's two halves and print its GMP records."""
    from conftest import golden
    g = golden("gaps_P337_d2310.json")
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    prog = tmp_path / "progress.txt"
    base = [str(cli), "-p", "337", "-d", "2310", "--mstart", "10000000", "--minc", "5000", "--max-prime", "100",
            "--min-merit", "5", "--sl", "7500", "--resume", str(prog), "-q"]
    subprocess.run(base + ["--ranges", "1"], capture_output=True, text=True, cwd=tmp_path, check=True)
    assert prog.read_text() == "337 2310 5000 10005000 1\n"
    subprocess.run(base + ["--ranges", "2"], capture_output=True, text=True, cwd=tmp_path, check=True)
    assert prog.read_text() == "337 2310 5000 10010000 2\n"
    assert (tmp_path / "records_337.txt").read_text().splitlines() == g["records"]


@pytest.mark.gpu
def test_cli_two_workers_print_ranges_in_order(pg, tmp_path):
    """--devices 0,0: two workers (two contexts on one device here; one per GPU on a multi-GPU node) take
    the two halves of the P=337 window; the records come out in m order and equal GMP's."""
    from conftest import golden
    g = golden("gaps_P337_d2310.json")
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    prog = tmp_path / "progress.txt"
    out = subprocess.run([str(cli), "-p", "337", "-d", "2310", "--mstart", "10000000", "--minc", "2500",
                          "--max-prime", "100", "--min-merit", "5", "--sl", "7500", "--ranges", "4",
                          "--devices", "0,0", "--resume", str(prog), "-q"],
                         capture_output=True, text=True, cwd=tmp_path, check=True).stdout
    import re
    rec = re.compile(r"^\d+ \d+\.\d{3} \d+ \* \d+# / \d+ - \d+$")
    assert [line for line in out.splitlines() if rec.match(line)] == g["records"]
    assert prog.read_text() == "337 2310 2500 10010000 4\n"


def test_cli_rejects_a_bad_device_list(pg):
    cli = pg.LIB_PATH.parent / "gap_search_gpu"
    r = subprocess.run([str(cli), "-p", "337", "-d", "2310", "--mstart", "1", "--minc", "10", "--max-prime", "1",
                        "--devices", "0,x"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stdout
