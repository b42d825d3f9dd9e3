"""The continuous-batching server (cuckoo-failure_b200/serve.py): every N_bad it serves, from
resident tables in a mix of requests, equals the same request computed alone (residues of its own
primes, then CRT).  CPU: the oracle stands behind a stand-in engine, with small chunks and a tiny
HBM budget so that chunks are grown, evicted and, when nothing fits, computed the plain way.  GPU:
the real engine."""
import os
import sys

import time

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import crt  # noqa: E402
import serve  # noqa: E402


class OracleTables:
    def __init__(self, primes, nmax, Fmax, d, model, delay):
        self.primes, self.nmax, self.Fmax, self.d, self.model = list(primes), nmax, max(nmax, Fmax), d, model
        self.polls_left = delay
        self.freed = False

    def close(self):
        self.freed = True


class OracleTicket:
    def __init__(self, rows, delay):
        self.rows, self.polls_left = rows, delay

    def done(self):
        self.polls_left -= 1
        return self.polls_left < 0

    def result(self):
        return self.rows


class OracleBackend:
    """The server's device side with the oracle behind it: builds become ready after
    `build_polls` readiness polls (a chunk in `slow` after many more), query results after
    `query_polls` polls, and plain requests run on a thread, like the GPU's worker."""

    def __init__(self, build_polls=2, query_polls=1, slow=(), slow_polls=40):
        import concurrent.futures as cf

        self.build_polls, self.query_polls, self.slow, self.slow_polls = build_polls, query_polls, set(slow), slow_polls
        self.pool = cf.ThreadPoolExecutor(1)
        self.built, self.queried = [], 0

    def build(self, primes, nmax, Fmax, d, model):
        c = cb.prime_range(0, 400).index(primes[0]) // len(primes)
        tab = OracleTables(primes, nmax, Fmax, d, model, self.slow_polls if (d, c) in self.slow else self.build_polls)
        self.built.append(tab)
        return tab

    @staticmethod
    def ready(tab):
        tab.polls_left -= 1
        return tab.polls_left < 0

    def query(self, tab, queries):
        assert not tab.freed and tab.polls_left < 0, "query on a table that is not ready or was freed"
        assert all(n <= tab.nmax and M <= tab.Fmax for n, M in queries)
        self.queried += 1
        rows = np.array([h.oracle_residues(p, max(n for n, _ in queries), tab.d, queries, tab.model)
                         for p in tab.primes], dtype=np.uint64)
        return OracleTicket(rows, self.query_polls)

    def plain(self, primes, n, M, d, model):
        return self.pool.submit(lambda: np.array([h.oracle_residues(p, n, d, [(n, M)], model)[0] for p in primes],
                                                 dtype=np.uint64))

    @staticmethod
    def free(tab):
        tab.close()


def pump_until_idle(srv, limit=10000):
    out = {}
    for _ in range(limit):
        for rid, res in srv.pump():
            out[rid] = res
        if srv.idle():
            return out
        time.sleep(0.0005)
    raise AssertionError("server did not finish")


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


def test_server_matches_requests_alone_with_eviction_and_plain_path():
    be = OracleBackend()
    budget = 6 * 4 * cb.tables_bytes(64, 160)  # room for a few small chunks of 4 primes only
    srv = serve.Server(be, budget, chunk=4)
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(18):
        n = int(rng.integers(8, 48))
        reqs.append((k, n, int(n * rng.uniform(1.5, 3.5)) + 1, int(rng.choice([2, 3]))))
    pc = crt.PrefixCRT(cb.prime_range(0, 64))
    got = {}
    for i in range(0, len(reqs), 6):  # three waves, each arriving while the last is in flight
        for rid, n, M, d in reqs[i:i + 6]:
            srv.submit(rid, n, M, d)
        for rid, res in srv.pump():
            got[rid] = res
    got.update(pump_until_idle(srv))
    for rid, n, M, d in reqs:
        assert len(got[rid]) >= cb.need(n, M, d)
        assert pc.crt(got[rid])[0] == alone(n, M, d), (rid, n, M, d)
    assert srv.builds > 0 and srv.used <= budget
    assert all(t.freed for t in be.built if t not in [c.tab for c in srv.chunks.values()])
    # a request far too large for the budget goes the plain way and is still exact
    big = serve.Server(OracleBackend(), 1, chunk=4)
    big.submit(0, 30, 70, 3)
    r = pump_until_idle(big)[0]
    assert pc.crt(r)[0] == alone(30, 70, 3) and big.plain == 1


def test_requests_are_answered_while_a_build_and_a_plain_request_are_in_flight():
    """A slow build of chunk (3, 1) and a plain request must not hold up the requests that ready
    chunks answer: those complete first, and every answer equals the request alone."""
    be = OracleBackend(slow=[(3, 1)], slow_polls=200)
    budget = 40 * 4 * cb.tables_bytes(64, 200)
    # tables for n > 36 cost more than the whole budget: such a request takes the plain path
    bytes_fn = lambda nmax, Fmax: budget + 1 if nmax > 36 else cb.tables_bytes(nmax, Fmax)
    srv = serve.Server(be, budget, chunk=4, bytes_fn=bytes_fn)
    pc = crt.PrefixCRT(cb.prime_range(0, 64))
    srv.submit("plain", 40, 90, 2)
    assert srv.pending["plain"].plain
    srv.submit("slow", 28, 60, 3)  # needs chunks 0 and 1 of d = 3: chunk 1 builds slowly
    order = []
    for k, (n, M, d) in enumerate([(10, 30, 2), (14, 25, 2), (9, 20, 2), (12, 40, 2)]):
        srv.submit(k, n, M, d)
    got = {}
    for _ in range(20000):
        for rid, res in srv.pump():
            got[rid] = res
            order.append(rid)
        if srv.idle():
            break
        time.sleep(0.0005)
    assert srv.idle()
    assert order.index("slow") > max(order.index(k) for k in range(4))
    for rid, (n, M, d) in [("plain", (40, 90, 2)), ("slow", (28, 60, 3)), (0, (10, 30, 2)), (1, (14, 25, 2)),
                           (2, (9, 20, 2)), (3, (12, 40, 2))]:
        assert pc.crt(got[rid])[0] == alone(n, M, d), rid


def test_a_chunk_too_small_is_replaced_when_old_and_new_do_not_fit_together():
    """A request that needs a resident chunk rebuilt larger, with room for the larger chunk but not
    for both: the small one is freed for it (no query on it in flight), and the request is answered."""
    be = OracleBackend()
    bytes_fn = lambda nmax, Fmax: 15 if nmax <= 64 else 20  # per prime: 480 / 640 bytes per chunk of 32
    srv = serve.Server(be, 1000, chunk=32, bytes_fn=bytes_fn)
    srv.submit(0, 20, 50, 2)
    r0 = pump_until_idle(srv)[0]
    assert srv.chunks[(2, 0)].nmax == 64
    srv.submit(1, 70, 150, 2)  # one chunk of 32 primes at n = 80
    r1 = pump_until_idle(srv)[1]
    pc = crt.PrefixCRT(cb.prime_range(0, 64))
    assert pc.crt(r0)[0] == alone(20, 50, 2) and pc.crt(r1)[0] == alone(70, 150, 2)
    assert srv.chunks[(2, 0)].nmax == 80 and srv.used <= 1000 and srv.plain == 0


def test_requests_above_the_resident_range_take_the_plain_path():
    be = OracleBackend()
    srv = serve.Server(be, 10**12, chunk=8, resident_nmax=24)
    srv.submit(0, 20, 50, 2)
    srv.submit(1, 30, 70, 2)
    got = pump_until_idle(srv)
    pc = crt.PrefixCRT(cb.prime_range(0, 64))
    assert pc.crt(got[0])[0] == alone(20, 50, 2) and pc.crt(got[1])[0] == alone(30, 70, 2)
    assert srv.plain == 1 and all(k[0] == 2 and ch.nmax <= 64 for k, ch in srv.chunks.items())


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
    """A short stream through the GPU backend with a budget that holds the small chunks only:
    builds, queries on ready chunks and plain rebuilds overlap; every N_bad equals the request
    computed alone."""
    stream = serve.poisson_stream(1.5, 40, 16, 700, seed=9)
    be = serve.GpuBackend(0)
    try:
        budget = 6 * 64 * cb.tables_bytes(320, 1280)
        lat, res, stats = serve.run(stream, be, budget, chunk=64, drain_s=180)  # a stall fails, never hangs
        with cb.Engine(0) as eng:
            for (t, n, M, d), x in zip(stream, res):
                ps = cb.prime_range(0, cb.need(n, M, d))
                r = eng.residues(ps, n, d, [(n, M)])
                assert x == crt.crt(list(zip(ps, (int(v) for v in r[:, 0]))))[0], (n, M, d)
    finally:
        be.close()
    assert stats["requests"] == len(stream) == stats["answered"] and all(v > 0 for v in lat)
    assert stats["plain"] > 0 and stats["builds"] > 0


def test_run_loop_with_crt_pool():
    """The timed loop end to end (continuous batching, spawn pool for CRT) with the oracle behind it."""
    stream = [(0.01 * k, n, M, d) for k, (n, M, d) in enumerate([(12, 30, 2), (20, 41, 3), (9, 20, 3), (30, 60, 2),
                                                                  (16, 40, 3), (25, 70, 2)])]
    lat, res, stats = serve.run(stream, OracleBackend(), 10**9, chunk=8)
    for (t, n, M, d), x in zip(stream, res):
        assert x == alone(n, M, d)
    assert stats["requests"] == 6 == stats["answered"] and all(v > 0 for v in lat)
    assert stats["residues_latency"]["p50_ms"] > 0
