"""Multi-GPU plan on CPU: gloo ranks, one disjoint m-window each, no data-path collective.

bench.py gives every rank its own window of m (rank_window, weak scaling);
ranks only meet for the barrier and the gather of their summaries, from which
aggregate() takes the whole job's m over the slowest rank's time.  Here two
gloo ranks run those functions of bench.py around an oracle search of their
windows: the gathered results must equal one search of the union, the windows
must be disjoint, every window must need the same operand width (so ranks run
the same kernel), and the aggregate must be the max-over-ranks figure.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    import time
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import oracle as O
    start, inc = bench.rank_window(rank, world)  # the product's own split of the m range
    t0 = time.perf_counter()
    with O.Job(503, 2190, 2_000, 200_000, threads=2) as j:
        ms = O.coprime_ms(start, 3_000, 2190)[:40]  # a slice of the rank's window keeps the CPU oracle fast
        prev, nxt = j.gmp_gaps(ms)
        bits = (j.K * (start + inc)).bit_length()
    dt = time.perf_counter() - t0 + rank  # this rank's time (rank 1 made the slowest)
    mine = {"dev_s": dt, "m": len(ms), "tests": 2 * len(ms), "e2e_s": 2 * dt, "launches": 3,
            "rank": rank, "window": [start, inc], "ms": ms.tolist(), "prev": prev.tolist(), "next": nxt.tolist(),
            "bits": bits}
    allr = bench.gather(dist, world, mine)  # bench.py's gather and aggregation, over gloo
    agg = bench.aggregate(allr)
    if rank == 0:
        out.put((allr, agg))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_m_range():
    """Two gloo ranks run bench.py's rank split (rank_window), gather and aggregate; each rank's gaps are
    GMP's (the oracle), the windows are disjoint and need the same operand width, the union equals one
    search, and the aggregate is the m of all ranks over the slowest rank's time."""
    import sys
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allr, agg = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = allr
    assert (a["rank"], b["rank"]) == (0, 1)
    assert a["window"][0] + a["window"][1] <= b["window"][0] or b["window"][0] + b["window"][1] <= a["window"][0]
    assert not set(a["ms"]) & set(b["ms"])                         # disjoint windows
    assert (a["bits"] + 31) // 32 == (b["bits"] + 31) // 32 == 22   # same operand width
    assert agg["dev_s"] == max(a["dev_s"], b["dev_s"]) == b["dev_s"]  # max over ranks
    assert agg["m"] == len(a["ms"]) + len(b["ms"]) and agg["value"] == agg["m"] / agg["dev_s"]
    assert agg["launches"] == 6 and agg["e2e_value"] == agg["m"] / (2 * b["dev_s"])
    union = np.array(sorted(a["ms"] + b["ms"]), dtype=np.uint64)
    with O.Job(503, 2190, 2_000, 200_000, threads=2) as j:
        prev, nxt = j.gmp_gaps(union)
    got = {m: (p, n) for g in allr for m, p, n in zip(g["ms"], g["prev"], g["next"])}
    assert [got[int(m)] for m in union] == list(zip(prev.tolist(), nxt.tolist()))


def test_rank_window_refuses_more_ranks_than_windows():
    import bench
    with pytest.raises(ValueError):
        bench.rank_window(0, len(bench.RANK_STARTS) + 1)
    with pytest.raises(ValueError):
        bench.rank_window(2, 2)
    assert bench.gather(None, 1, {"x": 1}) == [{"x": 1}]


def test_rank_windows_are_disjoint_and_22_words():
    import bench
    starts = bench.RANK_STARTS
    inc = bench.WORKLOAD["m_inc"]
    spans = sorted((s, s + inc) for s in starts)
    assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
    assert max(s + inc for s in starts) < 2 ** 21
