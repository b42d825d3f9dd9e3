"""The continuous-batching server (cuckoo-failure_b200/serve.py): every N_bad it serves, from
resident tables in a mix of requests, equals the same request computed alone (residues of its own
primes, then CRT).  CPU: the oracle stands behind a stand-in engine, with small chunks and a tiny
HBM budget so that chunks are grown, evicted and, when nothing fits, computed the plain way.  GPU:
the real engine."""
import os
import sys

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import crt  # noqa: E402
import serve  # noqa: E402


class OracleTables:
    def __init__(self, primes, nmax, Fmax, d, model):
        self.primes, self.nmax, self.Fmax, self.d, self.model = list(primes), nmax, max(nmax, Fmax), d, model

    def query(self, queries):
        return np.array([h.oracle_residues(p, max(n for n, _ in queries), self.d, queries, self.model)
                         for p in self.primes], dtype=np.uint64)

    def close(self):
        pass


class OracleEngine:
    def tables(self, primes, nmax, Fmax, d, model=0):
        return OracleTables(primes, nmax, Fmax, d, model)

    def residues(self, primes, nmax, d, queries, model=0):
        return np.array([h.oracle_residues(p, nmax, d, queries, model) for p in primes], dtype=np.uint64)


def alone(n, M, d, model=0):
    ps = cb.prime_range(0, cb.need(n, M, d, model))
    return crt.crt([(p, h.oracle_residues(p, n, d, [(n, M)], model)[0]) for p in ps])[0]


def test_grow_keeps_transform_length():
    for x in list(range(1, 3000, 7)) + [16384]:
        g = serve.grow(x)
        assert g >= x and cb.transform_length(g) == cb.transform_length(max(x, 64))


def test_stream_shape():
    st = serve.poisson_stream(5, 50, 64, 16384, seed=3)
    assert 150 < len(st) < 350 and all(64 <= n <= 16384 and M > n and d in (2, 3, 4) for _, n, M, d in st)
    assert [t for t, *_ in st] == sorted(t for t, *_ in st)


def test_rounds_match_requests_alone_with_eviction_and_plain_path():
    eng = OracleEngine()
    budget = 6 * cb.tables_bytes(64, 160)  # room for a few small chunks only
    srv = serve.Server(eng, budget, chunk=4)
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(18):
        n = int(rng.integers(8, 48))
        reqs.append((k, n, int(n * rng.uniform(1.5, 3.5)) + 1, int(rng.choice([2, 3]))))
    pc = crt.PrefixCRT(cb.prime_range(0, 64))
    got = {}
    for i in range(0, len(reqs), 6):  # three rounds
        got.update(srv.round(reqs[i:i + 6]))
    for rid, n, M, d in reqs:
        assert len(got[rid]) >= cb.need(n, M, d)
        assert pc.crt(got[rid])[0] == alone(n, M, d), (rid, n, M, d)
    assert srv.builds > 0 and srv.used <= budget
    # a request far too large for the budget goes the plain way and is still exact
    big = serve.Server(eng, 1, chunk=4)
    r = big.round([(0, 30, 70, 3)])[0]
    assert pc.crt(r)[0] == alone(30, 70, 3) and big.plain == 1


def test_prefix_crt_equals_pairwise_crt():
    import random

    ps = cb.prime_range(0, 300)
    pc = crt.PrefixCRT(ps)
    rng = random.Random(3)
    for k in (1, 2, 3, 7, 64, 100, 255, 256, 257, 300):
        rs = [rng.randrange(p) for p in ps[:k]]
        assert pc.crt(rs) == crt.crt(list(zip(ps[:k], rs)))


@pytest.mark.gpu
def test_served_results_equal_alone_on_gpu():
    stream = serve.poisson_stream(1.5, 40, 16, 400, seed=9)
    with cb.Engine(0) as eng:
        lat, res, stats = serve.run(stream, eng, 4e9, chunk=64)
        for (t, n, M, d), x in zip(stream, res):
            ps = cb.prime_range(0, cb.need(n, M, d))
            r = eng.residues(ps, n, d, [(n, M)])
            assert x == crt.crt(list(zip(ps, (int(v) for v in r[:, 0]))))[0], (n, M, d)
    assert stats["requests"] == len(stream) and all(v > 0 for v in lat)


def test_run_loop_with_crt_pool():
    """The timed loop end to end (continuous batching, spawn pool for CRT) with the oracle engine."""
    stream = [(0.01 * k, n, M, d) for k, (n, M, d) in enumerate([(12, 30, 2), (20, 41, 3), (9, 20, 3), (30, 60, 2),
                                                                  (16, 40, 3), (25, 70, 2)])]
    lat, res, stats = serve.run(stream, OracleEngine(), 10**9, chunk=8)
    for (t, n, M, d), x in zip(stream, res):
        assert x == alone(n, M, d)
    assert stats["requests"] == 6 and all(v > 0 for v in lat)
    assert stats["residues_latency"]["p50_ms"] > 0
