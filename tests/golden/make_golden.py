"""Generates the committed golden fixtures of tests/golden/ (run from the repo root):

    python tests/golden/make_golden.py

The reference ships no tests or known-answer vectors, so the fixtures come
from GMP 6.3.0 -- the library whose mpz_nextprime / mpz_prevprime /
mpz_probab_prime_p the reference calls on its CPU path (overflow.cpp:124-168)
-- through the CPU oracle, and every kind of fixture is cross-checked against
sympy, an independent implementation.

  prp_vectors.json   numbers with their strong base-2 verdict and GMP's
                     verdict: primes, composites, Carmichael numbers and
                     strong base-2 pseudoprimes (found here by brute force,
                     single- and multi-word)
  sieve_rows.json    sha256 of every sieve row of a P=337, d=2310 window,
                     plus a few full rows
  gaps_P*_d*.json    prev/next gaps from GMP for all m of the P=337 window
                     and seeded samples of the P=503, P=907 and P=3001 ones,
                     with the record lines above a merit threshold
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import random
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import numpy as np  # noqa: E402
import oracle as O  # noqa: E402
import sympy  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def merit(k_log: float, m: int, gap: int) -> float:
    import math
    return gap / (k_log + math.log(m))


def record(gap, mer, m, p, d, prev):
    return f"{gap} {mer:.3f} {m} * {p}# / {d} - {prev}"


def prp_vectors(rng: random.Random) -> dict:
    items = []

    def add(n: int, kind: str):
        items.append({"n": hex(n), "kind": kind, "bits": n.bit_length(),
                      "sprp2": O.prp(n, 1), "mr4": O.prp(n, 4), "gmp": O.probab_prime(n, 25)})

    for bits in (32, 64, 100, 128, 200, 256, 462, 512, 703, 768, 1024, 1264, 1536):
        for _ in range(3):
            p = int(sympy.nextprime(rng.getrandbits(bits) | (1 << (bits - 1))))
            add(p, "prime")
            c = p * int(sympy.nextprime(rng.getrandbits(24) | (1 << 23)))
            add(c, "composite")
            add(p + 2 if not sympy.isprime(p + 2) else p + 4, "odd")
    for n in (561, 1105, 1729, 2465, 2821, 6601, 8911, 41041, 62745, 825265):
        add(n, "carmichael")
    # strong base-2 pseudoprimes, brute force below 1e6
    small = [n for n in range(9, 1_000_000, 2) if O.prp(n, 1) == 1 and not sympy.isprime(n)]
    for n in small:
        add(n, "spsp2")
    # multi-word strong base-2 pseudoprimes of the forms p(2p-1), p(3p-2), p(4p-3)
    found = 0
    for bits in (40, 60, 100, 160, 250):
        tries = 0
        while tries < 400000:
            tries += 1
            p = int(sympy.nextprime(rng.getrandbits(bits) | (1 << (bits - 1))))
            for a, b in ((2, 1), (3, 2), (4, 3)):
                q = a * p - b
                n = p * q
                if O.prp(n, 1) == 1 and sympy.isprime(q):
                    add(n, "spsp2")
                    found += 1
            if found >= 2:
                found = 0
                break
    for it in items:  # sympy cross-check of the ground truth
        n = int(it["n"], 16)
        assert bool(it["gmp"]) == bool(sympy.isprime(n)), it
    return {"description": "strong PRP vectors; sprp2 = bases passed of the strong base-2 test, "
                           "mr4 = bases passed of 2,3,5,7, gmp = mpz_probab_prime_p(n, 25)",
            "gmp_version": O.gmp_version(), "items": items}


def sieve_rows() -> dict:
    P, d, sl, limit = 337, 2310, 7500, 1_000_000
    m_start, m_inc = 10_000_000, 2_000
    with O.Job(P, d, sl, limit) as j:
        ms = O.coprime_ms(m_start, m_inc, d)
        rows = j.sieve_m(ms)
        rows_x = j.sieve_x(m_start, m_inc)
        assert np.array_equal(rows, rows_x)
        # sympy spot check of a few bits
        for i in (0, len(ms) // 2, len(ms) - 1):
            m = int(ms[i])
            for idx in range(0, 2 * j.sly + 1, 997):
                y = idx - j.sly
                n = m * j.K + 2 * y
                comp = any(n % q == 0 for q in sympy.primerange(3, limit + 1))
                bit = (int(rows[i][idx >> 5]) >> (idx & 31)) & 1
                assert comp == bool(bit), (m, y)
        return {"P": P, "d": d, "sl": sl, "max_prime": limit, "m_start": m_start, "m_inc": m_inc,
                "words_per_m": int(rows.shape[1]),
                "ms": [int(m) for m in ms],
                "row_sha256": [hashlib.sha256(r.tobytes()).hexdigest() for r in rows],
                "full_rows": {str(int(ms[i])): [int(w) for w in rows[i]] for i in (0, 1, len(ms) - 1)}}


def gaps(name, P, d, m_start, m_inc, sl, limit, sample, min_merit, rng) -> dict:
    ms_all = O.coprime_ms(m_start, m_inc, d)
    ms = ms_all if sample is None else np.array(sorted(rng.sample(list(ms_all), sample)), dtype=np.uint64)
    with O.Job(P, d, sl, min(limit, 10**6)) as j:  # tables only matter for search(); gaps come from GMP
        prev, nxt = j.gmp_gaps(ms)
        k_log = j.K_log
        K = j.K
    for i in range(min(2, len(ms))):  # sympy cross-check
        c = int(ms[i]) * K
        assert int(sympy.nextprime(c)) - c == int(nxt[i]) and c - int(sympy.prevprime(c)) == int(prev[i])
    recs = []
    for m, a, b in zip(ms, prev, nxt):
        g = int(a) + int(b)
        mer = merit(k_log, int(m), g)
        if mer > min_merit:
            recs.append(record(g, mer, int(m), P, d, int(a)))
    return {"name": name, "P": P, "d": d, "m_start": m_start, "m_inc": m_inc, "sl": sl, "max_prime": limit,
            "k_log": k_log, "sampled": sample is not None, "min_merit": min_merit,
            "ms": [int(m) for m in ms], "prev_gap": [int(x) for x in prev], "next_gap": [int(x) for x in nxt],
            "records": recs}


def main():
    rng = random.Random(20261203)
    (OUT / "prp_vectors.json").write_text(json.dumps(prp_vectors(rng), indent=0))
    print("prp vectors done", flush=True)
    (OUT / "sieve_rows.json").write_text(json.dumps(sieve_rows()))
    print("sieve rows done", flush=True)
    windows = [
        ("gaps_P337_d2310.json", "P=337 d=2310 full window", 337, 2310, 10_000_000, 10_000, 7_500, 100_000_000, None, 5.0),
        ("gaps_P503_d2190.json", "P=503 d=2190 sample", 503, 2190, 1_000_000, 200_000, 10_000, 2_000_000_000, 48, 5.0),
        ("gaps_P907_d210.json", "P=907 d=210 sample", 907, 210, 1_000_000, 50_000, 18_000, 10_000_000_000, 24, 5.0),
        ("gaps_P3001_d2190.json", "P=3001 d=2190 sample", 3001, 2190, 1, 100_000, 40_000, 10_000_000_000, 6, 5.0),
    ]
    for fname, name, P, d, ms, mi, sl, lim, sample, mm in windows:
        (OUT / fname).write_text(json.dumps(gaps(name, P, d, ms, mi, sl, lim, sample, mm, rng)))
        print(fname, "done", flush=True)


if __name__ == "__main__":
    main()
