"""Multi-GPU plan on CPU: gloo ranks, one disjoint m-window each, no data-path collective.

bench.py gives every rank its own window of m (weak scaling); ranks only meet
for the barrier and the max-over-ranks time.  Here two gloo ranks each search
their window with the oracle and the gathered results must equal one search
of the union, the windows must be disjoint, and every window must need the
same operand width (so ranks run the same kernel).
"""
from __future__ import annotations

import os
import socket

import numpy as np
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
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import oracle as O
    start = bench.RANK_STARTS[rank]
    inc = 3_000  # a slice of each rank's window keeps the CPU oracle fast
    with O.Job(503, 2190, 2_000, 200_000, threads=2) as j:
        ms = O.coprime_ms(start, inc, 2190)
        prev, nxt = j.gmp_gaps(ms[:40])
        bits = (j.K * (start + bench.WORKLOAD["m_inc"])).bit_length()
    t = float(rank + 1)
    gathered = [None] * world
    dist.all_gather_object(gathered, {"rank": rank, "ms": ms[:40].tolist(), "prev": prev.tolist(),
                                      "next": nxt.tolist(), "bits": bits, "t": t})
    import torch
    tt = torch.tensor([t])
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((gathered, float(tt.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_m_range():
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
    gathered, tmax = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tmax == 2.0  # max over ranks
    a, b = gathered
    assert not set(a["ms"]) & set(b["ms"])                         # disjoint windows
    assert (a["bits"] + 31) // 32 == (b["bits"] + 31) // 32 == 22   # same operand width
    union = np.array(sorted(a["ms"] + b["ms"]), dtype=np.uint64)
    with O.Job(503, 2190, 2_000, 200_000, threads=2) as j:
        prev, nxt = j.gmp_gaps(union)
    got = {m: (p, n) for g in gathered for m, p, n in zip(g["ms"], g["prev"], g["next"])}
    assert [got[int(m)] for m in union] == list(zip(prev.tolist(), nxt.tolist()))


def test_rank_windows_are_disjoint_and_22_words():
    import bench
    starts = bench.RANK_STARTS
    inc = bench.WORKLOAD["m_inc"]
    spans = sorted((s, s + inc) for s in starts)
    assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
    assert max(s + inc for s in starts) < 2 ** 21
