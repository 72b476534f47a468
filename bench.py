"""Benchmark of the prime-gap search path on B200 (one JSON line on stdout).

Workload (the single-GPU configuration the metric is quoted on): P=503,
d=2190, every m in [1,000,000, 1,200,000) coprime to d (52,604 m), candidates
N = m*503#/2190 + X for X in [-10,000, 10,000] sieved by every prime <= 2e9,
strong base-2 PRP outward from X = 0 for the previous and the next prime,
records of merit > 22 with both primes confirmed by 16 strong bases.  A step
is one search of that window (sieve + PRP + finalize + record confirmation),
the inputs being the window bounds; the prime tables (98 M primes, 1.18 GB
with their K mod p and K^-1 residues) are read again by every step, far more
than the 126 MB L2, so no L2 flush is needed between steps.  Two windows are
in flight (two slots of the job, each with its own stream), each window's PRP
kernel holding at most 6 warps per SM, so one window's tail runs beside the
next window's sieve and search; `value` is the m of the K timed windows over
the device span from the first to the last of them.

Beside the headline the line carries (one GPU only): the other workloads --
P=337 / 1e8, P=907 / 1e10, a slice of P=3001 / 1e10 with its plain-form A/B
-- each window searched alone, and a short serving run (64 requests, Poisson
arrivals at 70% of the measured capacity, p50/p99 latency).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --serve      the full serving mix instead: capacity and p50/p99 latency

Under torchrun each rank searches its own window of 200,000 m (weak scaling,
no data-path collective); the reported time is the max over ranks.
`--impl reference` times the reference's CPU path on the host cores instead:
its per-X sieve walk up to its overflow cut, the PRP tests of the walk, and
GMP next / previous prime for the m left at the cut (the oracle's
restatement; the reference itself needs CGBN and primesieve).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(p=503, d=2190, m_start=1_000_000, m_inc=200_000, sl=10_000, max_prime=2_000_000_000,
                min_merit=22.0)
# distinct windows of 200,000 m per rank, all m < 2^21 so every rank runs the same 22-word operands
RANK_STARTS = [1_000_000, 1_200_000, 1_400_000, 1_600_000, 1_800_000, 800_000, 600_000, 400_000]
METRIC = "m/sec searched (prev+next prime of every m, bit-exact vs GMP)"
WINDOW_BITS = 5  # the reference's window for <= 1024-bit operands (gpu_testing.cu:50)


def workload_name(start: int, inc: int) -> str:
    return (f"P=503 d=2190 m in [{start:,}, {start + inc:,}) coprime to d, X in [-10000, 10000], "
            f"primes <= 2e9, merit > 22")


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (every 200 ms)."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------- CPU baseline

CPU_FRACTION = 0.005  # the reference's default --cpu-fraction (gap_common.h:47)


class CpuReference:
    """m/sec of the reference's CPU path for the workload window, on this host.

    The reference (gap_search_gpu.cpp:907-1006) walks the even X > 0 coprime to
    K's primes outward; for each X it sieves one row across every m of the
    window by every prime <= max_prime (gap_search_gpu.cpp:570-689, the
    corrected restatement of the oracle), PRP-tests the survivors among the m
    still without a next prime, and once fewer than cpu_fraction of the m
    remain (gap_search_gpu.cpp:976-997) hands those to GMP: next prime from
    m*K + X_cut + 1, previous prime when the next gap is long
    (overflow.cpp:145-160).  The PRP tests that the reference runs on its GPU
    are GMP strong base-2 tests here: this is the CPU path.

    Set-up (not timed): the cut X_cut -- the (1 - cpu_fraction) quantile of the
    next gaps of `gap_sample` seeded m, from GMP -- and the rows to walk (even X
    in [2, X_cut] with no factor among K's primes); the PRP tests per m of one
    side, from the oracle's search of `tests_sample` seeded m (half of its both-
    sided count).  A step (timed, all host threads): `rows` of the walk's rows
    sieved across the whole window (a different set each step), scaled to all
    of them; GMP strong tests on 24 candidates per thread, scaled to the walk's
    tests; GMP next and previous prime of `tail` of the sampled m with the
    longest next gaps, scaled to the cpu_fraction of the window left at the cut.
    """

    def __init__(self, threads: int, rows: int = 64, gap_sample: int = 2048, tests_sample: int = 32,
                 tail: int = 32, seed: int = 1):
        import random
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O  # the CPU restatement of the reference's path
        self.O, self.threads, self.rows, self.steps_done = O, threads, rows, 0
        W = WORKLOAD
        t0 = time.perf_counter()
        self.job = O.Job(W["p"], W["d"], W["sl"], W["max_prime"], threads=threads)
        self.ms_all = O.coprime_ms(W["m_start"], W["m_inc"], W["d"])
        rng = random.Random(seed)
        self.rng = rng
        sample = sorted(rng.sample(list(self.ms_all), gap_sample))
        _, nxt = self.job.gmp_gaps(sample)
        order = sorted(range(len(sample)), key=lambda i: int(nxt[i]))
        self.x_cut = int(nxt[order[int(math.ceil((1 - CPU_FRACTION) * len(sample))) - 1]])
        self.tail_ms = [sample[i] for i in order[-tail:]]
        kprimes = [q for q in range(3, W["p"] + 1, 2) if all(q % r for r in range(3, int(q ** 0.5) + 1, 2))
                   and W["d"] % q != 0]
        self.walk = [x // 2 for x in range(2, self.x_cut + 1, 2) if all(x % q for q in kprimes)]
        tsample = sorted(rng.sample(list(self.ms_all), tests_sample))
        _, _, _, tests = self.job.search(tsample, 1)
        self.tests_per_m = tests / (2 * len(tsample))  # one side: the reference's walk is next-side only
        self.setup_s = time.perf_counter() - t0

    def close(self):
        self.job.close()

    def step(self) -> dict:
        O, threads, W = self.O, self.threads, WORKLOAD
        sly = W["sl"] // 2
        R = min(self.rows, len(self.walk))
        n_walk = len(self.walk)
        ys = [self.walk[((i * n_walk) // R + self.steps_done) % n_walk] for i in range(R)]  # each step its own rows
        self.steps_done += 1
        t1 = time.perf_counter()
        self.job.sieve_x_rows(W["m_start"], W["m_inc"], ys)
        sieve_s = (time.perf_counter() - t1) * n_walk / R
        cands = [int(self.rng.choice(self.ms_all)) * self.job.K + 2 * self.rng.randrange(1, sly) + 1
                 for _ in range(threads * 24)]
        t2 = time.perf_counter()
        O.prp_batch(cands, 1, threads)
        per_test = (time.perf_counter() - t2) * threads / len(cands)  # one core's seconds per test
        n_m = len(self.ms_all)
        prp_s = n_m * self.tests_per_m * per_test / threads
        t3 = time.perf_counter()
        self.job.gmp_gaps(self.tail_ms)
        per_tail = (time.perf_counter() - t3) * threads / len(self.tail_ms)
        n_tail = CPU_FRACTION * n_m
        tail_s = n_tail * per_tail / max(1, min(threads, int(n_tail)))
        total = sieve_s + prp_s + tail_s
        return {"value": n_m / total, "unit": "m/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
                "sample": (f"reference walk of all {n_m} m: {R} of its {n_walk} sieve rows (even X in "
                           f"[2, {self.x_cut}] coprime to K; X_cut = next-gap quantile {1 - CPU_FRACTION} of "
                           f"2048 sampled m, the cpu_fraction {CPU_FRACTION} cut) timed across the window and "
                           f"scaled; {len(cands)} GMP strong base-2 tests timed ({per_test * 1e6:.1f} us/test/core)"
                           f" x {self.tests_per_m:.1f} tests/m; GMP next+prev prime of {len(self.tail_ms)} tail "
                           f"m timed, scaled to {n_tail:.0f} m"),
                "x_cut": self.x_cut, "walk_rows": n_walk, "rows_timed": R,
                "sieve_seconds_full": sieve_s, "prp_seconds_full": prp_s, "tail_seconds_full": tail_s,
                "prp_tests_per_sec": n_m * self.tests_per_m / total, "table_setup_seconds": self.setup_s}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------- GPU arm

def products_per_test(bits: int) -> int:
    """Limb products of one test by the fixed formula 2*L^2*(B + ceil(B/w)), L = ceil(B/32)."""
    L = (bits + 31) // 32
    return 2 * L * L * (bits + (bits + WINDOW_BITS - 1) // WINDOW_BITS)


def kernel_products_per_test(bits: int, limbs: int) -> int:
    """32x32->64 limb products the PRP kernel executes per strong base-2 test of a `bits`-bit number held in
    `limbs` words: bits - 1 Montgomery squarings, each L(L+1)/2 cross and diagonal products plus L*L reduction
    products and L quotient digits (base-2 multiplications are doublings: no products)."""
    L = limbs
    return (bits - 1) * (L * (L + 1) // 2 + L * L + L)


def traffic_per_launch() -> dict | None:
    f = ROOT / "profiles" / "ncu_traffic.json"
    if f.exists():
        try:
            return json.loads(f.read_text())
        except ValueError:
            return None
    return None


HBM_FALLBACK_GBS = 6650.0  # an earlier copy-bandwidth measurement on this pool's B200s


def hbm_peak() -> tuple[float, str]:
    """HBM copy bandwidth (GB/s) for the sieve's roofline and where it comes from."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            v = json.loads(f.read_text()).get("hbm_gbs")
            if v:
                return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except ValueError:
            pass
    return HBM_FALLBACK_GBS, "fallback (6.65 TB/s, an earlier copy measurement on this pool)"


def rank_window(rank: int, world: int, m_inc: int = WORKLOAD["m_inc"]) -> tuple[int, int]:
    """The m window of one rank: ranks search disjoint windows (weak scaling, no data-path exchange)."""
    if world > len(RANK_STARTS) or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}: at most {len(RANK_STARTS)} ranks")
    return RANK_STARTS[rank], m_inc


def gather(dist, world: int, mine: dict) -> list[dict]:
    """Every rank's summary on every rank (the only collective besides the barrier)."""
    if dist is None or world == 1:
        return [mine]
    allr = [None] * world
    dist.all_gather_object(allr, mine)
    return allr


def aggregate(allr: list[dict]) -> dict:
    """Whole-job figures from the ranks' summaries: m of all ranks over the slowest rank's device time."""
    dev_s = max(r["dev_s"] for r in allr)
    tot_m = sum(r["m"] for r in allr)
    return {"value": tot_m / dev_s, "dev_s": dev_s, "m": tot_m,
            "prp_tests_per_sec": sum(r["tests"] for r in allr) / dev_s,
            "e2e_value": tot_m / max(r["e2e_s"] for r in allr),
            "launches": sum(r["launches"] for r in allr)}


EXTRA = {  # the other workloads, each window searched alone on one GPU
    "P337": dict(p=337, d=2310, m_start=10_000_000, m_inc=10_000, sl=7_500, max_prime=100_000_000, min_merit=20.0,
                 windows=5),
    "P907": dict(p=907, d=210, m_start=1_000_000, m_inc=50_000, sl=18_000, max_prime=10_000_000_000,
                 min_merit=24.0, windows=3),
    # a slice of the P=3001 window (its first 600 m): 4 248-bit operands, plain-form A/B on the same m
    "P3001_slice": dict(p=3001, d=2190, m_start=1, m_inc=600, sl=40_000, max_prime=10_000_000_000,
                        min_merit=25.0, windows=2, plain=True, plain_windows=1),
}


def run_config(pg, ctx, w: dict) -> dict:
    """m/s of one workload window searched alone (device time of the search, inputs resident)."""
    job = pg.Job(w["p"], w["d"], w["sl"], w["max_prime"], max_m_inc=w["m_inc"], max_m=w["m_start"] + w["m_inc"],
                 confirm_merit=w["min_merit"], ctx=ctx)
    try:
        job.search(w["m_start"], w["m_inc"])  # warm-up (captures the window's graph)
        st = [job.search(w["m_start"], w["m_inc"]).stats for _ in range(w["windows"])]
        ms = statistics.median(x["total_ms"] for x in st)
        n = st[0]["m_count"]
        out = {"workload": f"P={w['p']} d={w['d']} m in [{w['m_start']:,}, {w['m_start'] + w['m_inc']:,}) coprime "
                           f"to d, X in [-{w['sl']}, {w['sl']}], primes <= {w['max_prime']:.0e}",
               "m": n, "ms_per_window": ms, "m_per_sec": n / (ms / 1e3),
               "prp_tests_per_sec": st[0]["prp_tests"] / (st[0]["total_ms"] / 1e3),
               "sieve_ms": statistics.median(x["sieve_ms"] for x in st), "limbs": job.info["limbs"],
               "tpi": job.info["tpi"], "windows_timed": len(st)}
        if w.get("plain"):
            pst = [job.search(w["m_start"], w["m_inc"], pg.PG_SEARCH_PLAIN).stats
                   for _ in range(w.get("plain_windows", w["windows"]))]
            pms = statistics.median(x["total_ms"] for x in pst)
            out["plain_ms_per_window"] = pms
            out["plain_m_per_sec"] = n / (pms / 1e3)
            out["batched_vs_plain"] = pms / ms
        return out
    finally:
        job.close()


PRP_SIZES = (512, 1024, 1536, 4352)  # the reference's BITS builds (gpu_state_and_checks, gpu_testing.cu:369-386)


def prp_rates(pg, ctx) -> dict:
    """Strong base-2 PRP tests per second of pg_prp_batch on random odd numbers of each operand size (one
    test per number, automatic layout), for comparison with the reference's per-size rates
    (gpu_testing.cu:65-100: 1 085 K PRP/s at 701#, ~1024 bits, TPI 8 on an A100)."""
    import numpy as np
    rng = np.random.default_rng(9)
    out = {}
    for bits in PRP_SIZES:
        words = bits // 32
        n = max(2048, (1 << 38) // (bits * bits))  # about the same device time at every size
        a = rng.integers(0, 2**32, size=(n, words), dtype=np.uint64).astype(np.uint32)
        a[:, 0] |= 1
        a[:, -1] = (a[:, -1] >> 2) | (1 << 29)  # bits - 2 bits: two spare bits for the lane-group layouts
        ctx.prp_words(a, 1)  # warm-up at full size: the context's buffers grow outside the timed call
        t = time.perf_counter()
        ctx.prp_words(a, 1)
        out[str(bits)] = {"numbers": n, "tests_per_sec": n / (time.perf_counter() - t)}
    return out


def run_ours(args, rank: int, world: int, local_rank: int, dist) -> dict | None:
    import torch
    import __graft_entry__
    pg = __graft_entry__.load_package()
    torch.cuda.set_device(local_rank)
    W = WORKLOAD
    m_start, m_inc = rank_window(rank, world, args.m_inc)
    ctx = pg.Context(local_rank)
    # autotune (pg_autotune_ex) on this rank's window: threads per number, sieve tile bound, PRP warps per SM
    tune = None
    knobs = {}
    if not args.no_tune:
        t0 = time.perf_counter()
        tune = pg.autotune_ex(W["p"], W["d"], W["sl"], W["max_prime"], m_start, m_inc, ctx=ctx, reps=2,
                              confirm_merit=W["min_merit"])
        tune["seconds"] = time.perf_counter() - t0
        knobs = {k: tune["knobs"][k] for k in ("small_limit", "tpi")}
        if args.warps_per_sm is None:
            args.warps_per_sm = tune["warps_per_sm"]
    if args.warps_per_sm is None:
        args.warps_per_sm = 6
    t0 = time.perf_counter()
    job = pg.Job(W["p"], W["d"], W["sl"], W["max_prime"], max_m_inc=m_inc, max_m=max(RANK_STARTS) + m_inc,
                 rounds=1, confirm_merit=W["min_merit"], ctx=ctx, **knobs)
    setup_s = time.perf_counter() - t0
    imad_peak = ctx.imad_peak()
    dev = torch.device("cuda", local_rank)
    streams = [torch.cuda.ExternalStream(job.stream_ptr(k), device=dev) for k in range(pg.PG_SEARCH_SLOTS)]

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def pipelined(steps: int, sampler: bool, records: bool):
        """`steps` windows with PG_SEARCH_SLOTS in flight; device span from CUDA
        events on the slot streams, plus the host wall clock of the same calls."""
        barrier()
        clk = ClockSampler(local_rank) if sampler else None
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(streams[0])
        for st in streams[1:]:
            st.wait_event(ev0)
        t0 = time.perf_counter()
        stats, pending, nrec, res = [], [], 0, None
        for i in range(steps):
            pending.append(job.submit(m_start, m_inc, pg.PG_SEARCH_PERSISTENT,
                                      ((pg.PG_SUBMIT_DRAIN | (args.drain << 8)) if args.drain else 0)
                                      | (args.warps_per_sm << 16)))
            while len(pending) == pg.PG_SEARCH_SLOTS or (i == steps - 1 and pending):
                res = job.wait(pending.pop(0))
                stats.append(res.stats)
                if records:
                    nrec += len(job.records(res, W["min_merit"]))
        wall = time.perf_counter() - t0
        for st in streams[1:]:
            e = torch.cuda.Event()
            e.record(st)
            streams[0].wait_event(e)
        ev1.record(streams[0])
        torch.cuda.synchronize()
        span_ms = ev0.elapsed_time(ev1)
        clocks = clk.stop() if clk else None
        barrier()
        return res, stats, span_ms, wall, nrec, clocks

    def synchronous(form: int, steps: int):
        barrier()
        stats = []
        for _ in range(steps):
            stats.append(job.search(m_start, m_inc, form).stats)
        barrier()
        return stats

    pipelined(args.warmup, False, False)
    res, stats, span_ms, _, _, clocks = pipelined(args.steps, True, False)
    m_count = stats[0]["m_count"]
    # each window alone (no overlap): the PRP kernel's and the sieve's own times for the rooflines
    sstats = synchronous(pg.PG_SEARCH_PERSISTENT, args.steps)
    kern_ms = sum(s["search_kernel_ms"] for s in sstats)
    tests = sum(s["prp_tests"] for s in sstats)
    sync_ms = sum(s["total_ms"] for s in sstats) / args.steps
    sieve_ms = statistics.median(s["sieve_ms"] for s in sstats)
    survivors = sstats[0]["survivors"]
    # plain form, same window (the batched-vs-plain A/B)
    plain = None
    if not args.no_plain:
        job.search(m_start, m_inc, pg.PG_SEARCH_PLAIN)
        pstats = synchronous(pg.PG_SEARCH_PLAIN, args.steps)
        pdev = sum(s["total_ms"] for s in pstats)
        plain = {"ms_per_step": pdev / args.steps, "m_per_sec": m_count * args.steps / (pdev / 1e3),
                 "prp_tests": pstats[0]["prp_tests"], "passes": pstats[0]["passes"],
                 "kernel_launches_per_step": pstats[0]["kernel_launches"]}
    # end to end through the public API: host window in, host gaps + confirmed records out
    _, e2e_stats, _, e2e_s, nrec, _ = pipelined(args.steps, False, True)
    # bit-exactness self-check of this run against the committed GMP fixture
    exact = None
    if rank == 0:
        gold = json.loads((ROOT / "tests" / "golden" / "gaps_P503_d2190.json").read_text())
        pos = {int(m): i for i, m in enumerate(res.ms)}
        exact = all((int(res.prev_gap[pos[m]]), int(res.next_gap[pos[m]])) == (a, b)
                    for m, a, b in zip(gold["ms"], gold["prev_gap"], gold["next_gap"]) if m in pos)
    mine = {"dev_s": span_ms / 1e3, "kern_s": kern_ms / 1e3, "tests": sum(s["prp_tests"] for s in stats),
            "m": m_count * args.steps, "e2e_s": e2e_s, "clocks": clocks, "sync_ms": sync_ms,
            "launches": sum(s["kernel_launches"] for s in stats)}
    allr = gather(dist, world, mine)
    if rank != 0:
        job.close()
        ctx.close()
        return None
    agg = aggregate(allr)
    bits = (job.K * (m_start + m_inc // 2)).bit_length()
    limbs = job.info["limbs"]
    ppt_formula = products_per_test(bits)
    ppt = kernel_products_per_test(bits, limbs)
    kern_s = kern_ms / 1e3
    peak = imad_peak / 2                               # a 32x32->64 product needs a lo and a hi multiply-add
    tr = traffic_per_launch()
    roof = {"bound": "imad", "achieved": tests * ppt / kern_s / 1e9, "peak": peak / 1e9,
            "unit": "G limb-products/s", "frac": tests * ppt / kern_s / peak,
            "frac_formula": tests * ppt_formula / kern_s / peak,
            "traffic": tr.get("bytes_per_launch") if tr else None,
            "imad_pipe_busy_ncu": tr.get("imad_pipe_busy") if tr else None,
            "kernel": f"k_search_persistent<{limbs}>",
            "work": f"{ppt} limb products per {bits}-bit test ({bits - 1} squarings of {limbs} words: "
                    f"L(L+1)/2 + L^2 + L each), {tests // args.steps} tests per launch; frac_formula uses the "
                    f"fixed 2*L^2*(B+ceil(B/5)) = {ppt_formula}",
            "peak_source": "in-run microbenchmark (pg_measure_imad_peak: 32-bit IMAD/s / 2); "
                           "MEASURED_PEAKS.json has no integer-multiply figure"}
    hbm, hbm_src = hbm_peak()
    esz = 8 if W["max_prime"] >= 2 ** 32 else 4
    table_b = job.info["num_primes"] * 3 * esz
    walk_b = job.info["num_primes"] * 8 if W["max_prime"] < 2 ** 32 else 0  # sa, sb of every large prime
    rows_b = m_count * job.info["words_per_m"] * 4
    sieve_b = table_b + walk_b + 2 * rows_b + survivors * 2
    sieve = {"bound": "hbm", "achieved": sieve_b / (sieve_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
             "frac": sieve_b / (sieve_ms / 1e3) / 1e9 / hbm, "ms_per_window": sieve_ms,
             "bytes_per_window": sieve_b,
             "work": f"prime table {table_b / 1e9:.3f} GB ({job.info['num_primes']} primes x 3 x {esz} B, read "
                     f"once) + walk table {walk_b / 1e9:.3f} GB (2 x u32 per prime, read once) + rows "
                     f"{rows_b / 1e6:.1f} MB written and read once + {survivors} survivors x 2 B; "
                     "time = sieve kernels of a window alone (large-prime search, small-prime tiles and lists)",
             "peak_source": hbm_src}
    line = {
        "metric": METRIC, "value": agg["value"], "unit": "m/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": agg["dev_s"] * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name(RANK_STARTS[0], m_inc),
                   "form": ("autotuned " if tune else "") + f"persistent, {pg.PG_SEARCH_SLOTS} windows in flight"
                           + (f", {args.warps_per_sm} PRP warps per SM per window" if args.warps_per_sm else "")
                           + (f", draining to {args.drain} lanes per unresolved side" if args.drain else "")
                           + ", records confirmed with 16 bases",
                   "m_per_gpu_per_step": m_count, "sl": W["sl"], "max_prime": W["max_prime"],
                   "limbs": limbs, "tpi": job.info["tpi"], "small_limit": job.params.small_limit or 65536,
                   "warps_per_sm": args.warps_per_sm, "parallelism": f"weak: {world} disjoint m-windows",
                   "l2": "inputs larger than L2 (1.18 GB prime tables read every step)"},
        "prp_tests_per_sec": agg["prp_tests_per_sec"],
        "ms_per_step_one_window_alone": max(r["sync_ms"] for r in allr),
        "setup_seconds": setup_s,
        "bit_exact_vs_gmp_sample": exact,
        "autotune": tune,
        "roofline": roof,
        "sieve": sieve,
        "e2e": {"value": agg["e2e_value"], "unit": "m/s",
                "h2d_bytes_per_step": stats[0]["h2d_bytes"], "d2h_bytes_per_step": stats[0]["d2h_bytes"],
                "records_per_step": nrec / max(1, args.steps),
                "confirm_tests_per_step": sum(x["confirm_tests"] for x in e2e_stats) / max(1, args.steps)},
        "gpu_launches": agg["launches"],
        "clocks": allr[0]["clocks"],
    }
    if plain is not None:
        line["plain"] = plain
        line["batched_vs_plain"] = agg["value"] / (plain["m_per_sec"] * world)
    job.close()
    if world == 1 and not args.no_extra:
        line["configs"] = {name: run_config(pg, ctx, w) for name, w in EXTRA.items()}
        line["configs"]["prp_rates"] = prp_rates(pg, ctx)
        ctx.close()
        line["configs"]["serving"] = run_serve(args, n_jobs=64, compact=True, preempt=0)
        line["configs"]["serving_preempt"] = run_serve(args, n_jobs=64, compact=True, preempt=SERVE_PREEMPT_US,
                                                       rate=line["configs"]["serving"]["arrival_rate_jobs_per_s"])
        line["configs"]["serving_preempt"]["arrival_rate_source"] = "the rate of configs.serving (same load)"
    else:
        ctx.close()
    if world == 1 and not args.no_cpu:
        ref = CpuReference(host_threads())
        try:
            line["cpu_baseline"] = ref.step()
        finally:
            ref.close()
    return line


def run_reference(args) -> dict:
    threads = host_threads()
    ref = CpuReference(threads, rows=24)  # 24 rows a step, shifted by one row per step
    vals, last = [], None
    try:
        for i in range(args.warmup + args.steps):
            est = ref.step()
            if i >= args.warmup:
                vals.append(est["value"])
                last = est
    finally:
        ref.close()
    v = statistics.median(vals)
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "m/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": workload_name(WORKLOAD["m_start"], WORKLOAD["m_inc"]),
                       "implementation": "CPU restatement of the reference path (oracle/, GMP 6.3.0): its per-X "
                                         "sieve walk to the cpu_fraction cut, GMP PRP tests, GMP next/prev prime "
                                         "of the tail; the reference needs CGBN and primesieve, absent here"},
            "cpu_baseline": {**{k: last[k] for k in ("unit", "cores", "kind", "sample", "cpu")}, "value": v},
            "e2e": {"value": v, "unit": "m/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "prp_tests_per_sec": last["prp_tests_per_sec"]}


# ----------------------------------------------------------- serving

SERVE_SEED = 4
SERVE_PREEMPT_US = 20_000  # a launch running 20 ms yields to windows that have waited as long


def serve_requests(n: int = 256, seed: int = SERVE_SEED, limit: int = 1_000_000_000) -> list[tuple]:
    """The serving mix: n requests, P in {337, 503, 907}, d in {210, 2190,
    2310}, windows of 500-20,000 m starting uniformly in [1e6, 1e9],
    SL = round(8 ln N) with N = m_start * P#/d, sieve limit 1e9."""
    import numpy as np
    import __graft_entry__
    pg = __graft_entry__.load_package()
    rng = np.random.default_rng(seed)
    primorial = {}
    for P in (337, 503, 907):
        k = 1
        for q in range(2, P + 1):
            if all(q % r for r in range(2, int(q ** 0.5) + 1)):
                k *= q
        primorial[P] = k
    out = []
    for _ in range(n):
        P = int(rng.choice([337, 503, 907]))
        d = int(rng.choice([210, 2190, 2310]))
        inc = int(rng.integers(500, 20_001))
        start = int(rng.integers(1_000_000, 1_000_000_001))
        sl = round(8 * (pg.k_log_of(primorial[P] // d) + math.log(start)))
        out.append((P, d, sl, limit, start, inc))
    return out


def run_serve(args, n_jobs: int | None = None, compact: bool = False, preempt: int | None = None,
              rate: float | None = None) -> dict:
    """Capacity (all requests queued at once) and latency under Poisson
    arrivals at 70% of that capacity, through pg_server_*.  compact: the
    short run of the default bench line (n_jobs requests, the server's
    default launch shape); preempt: the server's preempt_us (None = the
    --serve-preempt-us option); rate: the arrival rate to use instead (so
    two servers are compared at one load)."""
    import threading
    import numpy as np
    import __graft_entry__
    pg = __graft_entry__.load_package()
    reqs = serve_requests(n_jobs or args.serve_jobs)
    classes = sorted({(p, d) for p, d, *_ in reqs})
    max_sl = max(r[2] for r in reqs)
    wps = 0 if compact else args.warps_per_sm
    batch_m = 0 if compact else args.serve_batch_m
    slots = 0 if compact else args.serve_slots
    preempt_us = preempt if preempt is not None else args.serve_preempt_us
    with pg.Server(0, max_sl=max_sl, warps_per_sm=wps, batch_m=batch_m, slots=slots, preempt_us=preempt_us) as srv:
        # resident tables for every (P, d) first: one small request per class
        warm = [srv.submit(p, d, 1_000, reqs[0][3], 1_000_001, 200) for p, d in classes]
        t = time.perf_counter()
        for i in warm:
            srv.wait(i)
        table_s = time.perf_counter() - t
        # closed loop: every request at once
        t0 = srv.clock()
        ids = [srv.submit(p, d, sl, lim, m0, inc) for p, d, sl, lim, m0, inc in reqs]
        infos = [srv.wait(i).info for i in ids]
        span = max(x["done_s"] for x in infos) - t0
        m_total = sum(x["m_count"] for x in infos)
        cap_jobs = len(reqs) / span
        st_closed = srv.stats()
        # open loop: Poisson arrivals at 70% of capacity (or at the given rate)
        rate_source = "the given rate" if rate else ("--serve-rate" if args.serve_rate > 0 else "70% of capacity")
        rate = rate or (args.serve_rate if args.serve_rate > 0 else 0.7 * cap_jobs)
        gaps = np.random.default_rng(SERVE_SEED + 1).exponential(1.0 / rate, len(reqs))
        arrivals = np.cumsum(gaps)
        ids2 = [None] * len(reqs)

        def feeder():
            base = time.perf_counter()
            for k, r in enumerate(reqs):
                delay = arrivals[k] - (time.perf_counter() - base)
                if delay > 0:
                    time.sleep(delay)
                ids2[k] = srv.submit(*r)

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        infos2 = [srv.wait(i).info for i in ids2]
        lat = np.array([x["done_s"] - x["submit_s"] for x in infos2]) * 1e3
        wait = np.array([x["start_s"] - x["submit_s"] for x in infos2]) * 1e3  # until its first window is placed
        st = srv.stats()
        by_p = {}
        for P in sorted({r[0] for r in reqs}):
            sel = np.array([r[0] == P for r in reqs])
            by_p[str(P)] = {"n": int(sel.sum()), "p50_ms": round(float(np.percentile(lat[sel], 50)), 1),
                            "p99_ms": round(float(np.percentile(lat[sel], 99)), 1),
                            "placed_p50_ms": round(float(np.percentile(wait[sel], 50)), 1),
                            "placed_p99_ms": round(float(np.percentile(wait[sel], 99)), 1)}
    return {
        "metric": f"serving latency p99 ({len(reqs)} gap-search requests, Poisson arrivals at {rate:.1f}/s)",
        "arrival_rate_source": rate_source,
        "value": round(float(np.percentile(lat, 99)), 2), "unit": "ms", "higher_is_better": False,
        "p50_ms": round(float(np.percentile(lat, 50)), 2), "p99_ms": round(float(np.percentile(lat, 99)), 2),
        "mean_ms": round(float(lat.mean()), 2), "latency_by_P": by_p,
        "capacity_jobs_per_s": round(cap_jobs, 2), "capacity_m_per_s": round(m_total / span, 1),
        "arrival_rate_jobs_per_s": round(rate, 2), "closed_loop_s": round(span, 3),
        "table_build_s": round(table_s, 3),
        "launches": st_closed["launches"], "windows": st_closed["windows"],
        "prp_tests_closed": st_closed["prp_tests"], "sieve_ms_closed": round(st_closed["sieve_ms"], 1),
        "prp_ms_closed": round(st_closed["prp_ms"], 1), "peak_bytes": st["peak_bytes"],
        "n_gpus": 1, "data": "synthetic (seeded request mix)",
        "config": {"workload": f"{len(reqs)} requests, P in {{337,503,907}}, d in {{210,2190,2310}}, "
                               "500-20000 m from [1e6,1e9], SL=round(8 ln N), primes <= 1e9",
                   "seed": SERVE_SEED, "warps_per_sm": wps, "batch_m": batch_m or 65536,
                   "slots": slots or (4 if preempt_us else 2), "preempt_us": preempt_us},
        "preemptions": st["preemptions"],
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form A/B")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other workloads and the short serving run (one GPU only)")
    ap.add_argument("--drain", type=int, default=0, metavar="D",
                    help="let the PRP kernel's warps leave as a window drains, keeping D lanes per "
                         "unresolved side (PG_SUBMIT_DRAIN; 0 = off)")
    ap.add_argument("--warps-per-sm", type=int, default=None, metavar="W",
                    help="cap each launch's PRP kernel at W resident warps per SM so the two launches "
                         "in flight run side by side (0 = as many as fit; default: the autotuner's choice for "
                         "the window benchmark, 6 with --no-tune, and 0 for --serve, whose launches are "
                         "large enough that the cap costs more than it saves)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (default knobs: automatic threads per number, 65536 sieve tile "
                         "bound, 6 warps per SM)")
    ap.add_argument("--m-inc", type=int, default=WORKLOAD["m_inc"],
                    help="m per window (default 200000; smaller windows are for profiling only)")
    ap.add_argument("--serve", action="store_true",
                    help="the serving workload instead: p50/p99 latency of a request mix (pg_server_*)")
    ap.add_argument("--serve-jobs", type=int, default=256)
    ap.add_argument("--serve-batch-m", type=int, default=0,
                    help="coprime m per search launch of the server (0 = its default, 65536)")
    ap.add_argument("--serve-slots", type=int, default=0, help="server launch slots (0 = its default: 2, 4 with preemption)")
    ap.add_argument("--serve-preempt-us", type=int, default=0,
                    help="server preemption (pg_server_params.preempt_us; 0 = off)")
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="arrival rate in requests/s for the latency run (0 = 70%% of the measured capacity)")
    args = ap.parse_args(argv)
    if args.warps_per_sm is None and args.serve:
        args.warps_per_sm = 0
    if args.serve:
        print(json.dumps(run_serve(args)), flush=True)
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return 0
    if world > len(RANK_STARTS):
        raise SystemExit(f"at most {len(RANK_STARTS)} ranks")
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dd
        torch.cuda.set_device(local_rank)
        dd.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                              device_id=torch.device("cuda", local_rank))
        dist = dd
    try:
        line = run_ours(args, rank, world, local_rank, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
