#!/usr/bin/env python3
"""Continuous-batching query server over resident suffix tables.

A request nbad(n, M, d) is answered as the reference answers it: N_bad modulo the first
need(n, M, d) primes of the fixed list (fast/cuckoo_fast.cu:403-459), recombined by CRT
(crt.py, the fast/post_gmp.py step).  The reference rebuilds a suffix table per prime for every
run.  This server keeps the tables on the GPU across requests (cf_tables_*), per (d, model) in
prime chunks of CHUNK primes, each chunk built to some (n, F) and answering any later request
with n' <= n, M' <= F in O(n'^2) per prime.  A chunk is built, or rebuilt larger, only when a
request needs more than it holds; chunks are admitted under an HBM budget and evicted least
recently used.

Each round of the loop takes every request that has arrived (continuous batching: requests
arriving while the GPU works join the next round), builds the chunks the round is missing, and
answers all of the round's requests per chunk with one query launch.  A request whose tables
cannot be resident within the budget is computed the plain way (cf_residues, no residency) in
its round.  The residues of a served request cover whole chunks (the primes beyond its need
change nothing: N_bad is below the product of its own primes), so every CRT is over a prefix of
the list whose length is a multiple of the chunk, and a pool of host processes (crt.PrefixCRT,
constants cached at start) recombines them while the GPU serves the next round.  Two latencies
are kept per request, from its arrival: residues ready, and N_bad ready.

    python cuckoo-failure_b200/serve.py [--seconds 10] [--rate 200] [--nmax 2048] [--budget-gb 150] [--seed 1]
"""
import argparse
import math
import os
import sys
import time
from collections import OrderedDict

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import crt  # noqa: E402
import cuckoo_b200 as cb  # noqa: E402

CHUNK = 256  # primes per resident table set


def poisson_stream(seconds, rate, n_lo, n_hi, seed, d_choices=(2, 3, 4), m_ratio=(1.5, 4.0)):
    """Seeded request stream: exponential gaps at `rate` per second, n log-uniform in [n_lo, n_hi],
    M = round(n U[m_ratio]) (> n), d uniform in d_choices.  Returns [(arrival_s, n, M, d)]."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return out
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        M = max(n + 1, int(round(n * rng.uniform(*m_ratio))))
        d = int(rng.choice(d_choices))
        out.append((t, n, M, d))


def grow(x, lo=64):
    """Table size for a request of size x: the least 2^k m / 8 (m = 5..8) >= max(x, lo), so a run
    of slightly larger requests rebuilds rarely and no size crosses a power of two (the transform
    length) that x itself does not."""
    x = max(x, lo)
    k = max(0, (x - 1).bit_length() - 1)  # 2^k < x <= 2^(k+1) (x > 1)
    for m in (5, 6, 7, 8):
        s = (m << (k + 1)) // 8
        if s >= x:
            return s
    return 1 << (k + 1)


class Server:
    def __init__(self, engine, budget_bytes, model=cb.MODEL_SUBSET, n_cap=16384, chunk=CHUNK):
        self.eng, self.budget, self.model, self.n_cap, self.chunk = engine, budget_bytes, model, n_cap, chunk
        self.chunks = OrderedDict()  # (d, chunk index) -> Tables, in LRU order
        self.used = 0
        self.builds = 0
        self.plain = 0

    def _bytes(self, tab):
        return len(tab.primes) * cb.tables_bytes(tab.nmax, tab.Fmax)

    def _evict_for(self, need_bytes, keep):
        for key in list(self.chunks):
            if self.used + need_bytes <= self.budget:
                break
            if key in keep:
                continue
            tab = self.chunks.pop(key)
            self.used -= self._bytes(tab)
            tab.close()
        return self.used + need_bytes <= self.budget

    def _ensure(self, d, c, n, M, keep):
        """Chunk c of degree d resident with n and M covered; False if the budget forbids it."""
        tab = self.chunks.get((d, c))
        if tab is not None and tab.nmax >= n and tab.Fmax >= M:
            self.chunks.move_to_end((d, c))
            return True
        n2 = min(self.n_cap, max(grow(n), tab.nmax if tab else 0))
        F2 = max(grow(M), tab.Fmax if tab else 0, n2)
        cnt = self.chunk
        size = cnt * cb.tables_bytes(n2, F2)
        if tab is not None:
            self.chunks.pop((d, c))
            self.used -= self._bytes(tab)
            tab.close()
        if not self._evict_for(size, keep):
            return False
        primes = cb.prime_range(c * cnt, cnt)
        self.chunks[(d, c)] = self.eng.tables(primes, n2, F2, d, model=self.model)
        self.used += size
        self.builds += 1
        return True

    def round(self, reqs):
        """Residues for a batch of requests [(id, n, M, d)] -> {id: [residue modulo prime i, i = 0, 1, ...]}
        covering at least the request's need(n, M, d) primes (whole chunks when served resident)."""
        res = {rid: {} for rid, _, _, _ in reqs}
        plain = []
        # which chunks each request needs
        need = {rid: cb.need(n, M, d, self.model) for rid, n, M, d in reqs}
        uses = {}
        for rid, n, M, d in reqs:
            for c in range((need[rid] + self.chunk - 1) // self.chunk):
                uses.setdefault((d, c), []).append((rid, n, M))
        keep = set(uses)
        resident = {}
        for (d, c), items in uses.items():
            n = max(x[1] for x in items)
            M = max(x[2] for x in items)
            resident[(d, c)] = self._ensure(d, c, n, M, keep)
        bad = {rid for (d, c), items in uses.items() if not resident[(d, c)] for rid, _, _ in items}
        for (d, c), items in uses.items():
            items = [x for x in items if x[0] not in bad]
            if not items:
                continue
            tab = self.chunks[(d, c)]
            out = tab.query([(n, M) for _, n, M in items])
            for jj, (rid, n, M) in enumerate(items):
                res[rid][c] = out[:, jj].tolist()  # primes c*chunk .. c*chunk + chunk - 1
        for rid, n, M, d in reqs:
            if rid in bad:
                plain.append((rid, n, M, d))
        for rid, n, M, d in plain:  # no residency: rebuild for this request alone
            ps = cb.prime_range(0, need[rid])
            r = self.eng.residues(ps, n, d, [(n, M)], model=self.model)
            res[rid] = {0: r[:, 0].tolist()}
            self.plain += 1
        return {rid: [x for c in sorted(v) for x in v[c]] for rid, v in res.items()}


# ---- host CRT workers (separate processes, started with spawn) ----
_PCRT = None


def _crt_init(primes, warm_lengths):
    global _PCRT
    _PCRT = crt.PrefixCRT(primes)
    for k in warm_lengths:
        _PCRT.crt([0] * k)


def _crt_job(residues):
    return _PCRT.crt(residues)[0]


def crt_pool(max_primes, chunk=CHUNK, workers=None):
    """Process pool whose workers hold crt.PrefixCRT over the fixed list, its constants for every
    chunk-multiple prefix computed before the pool is returned."""
    import concurrent.futures as cf
    import multiprocessing as mp

    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    kmax = ((max_primes + chunk - 1) // chunk) * chunk
    primes = [int(p) for p in cb.prime_range(0, kmax)]
    warm = list(range(chunk, kmax + 1, chunk))
    pool = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                  initializer=_crt_init, initargs=(primes, warm))
    list(pool.map(time.sleep, [0.05] * (2 * workers)))  # every worker started and warm
    return pool


def run(stream, engine, budget_bytes, model=cb.MODEL_SUBSET, warm=None, max_round=512, chunk=CHUNK, pool=None):
    """Serve a timed stream [(arrival_s, n, M, d)] in real time.  `warm`, if given, is a list of
    (n, M, d) built before the clock starts.  Returns (latencies_s, results, stats): the latency to
    N_bad per request, N_bad per request, and counters including the latency to residues."""
    srv = Server(engine, budget_bytes, model, chunk=chunk)
    for n, M, d in warm or []:
        for c in range((cb.need(n, M, d, model) + chunk - 1) // chunk):
            srv._ensure(d, c, n, M, set())
    own_pool = pool is None
    if own_pool:
        kmax = max([cb.need(n, M, d, model) for _, n, M, d in stream] + [1])
        pool = crt_pool(kmax, chunk)
    futs = [None] * len(stream)
    lat, res_lat = [0.0] * len(stream), [0.0] * len(stream)
    t0 = time.perf_counter()
    gpu_s, rounds, i = 0.0, 0, 0

    def stamp(k):
        def cb_(_f):
            lat[k] = time.perf_counter() - t0 - stream[k][0]
        return cb_

    while i < len(stream):
        now = time.perf_counter() - t0
        if stream[i][0] > now:
            time.sleep(min(stream[i][0] - now, 0.005))
            continue
        j = i
        while j < len(stream) and stream[j][0] <= now and j - i < max_round:
            j += 1
        batch = [(k, stream[k][1], stream[k][2], stream[k][3]) for k in range(i, j)]
        g0 = time.perf_counter()
        out = srv.round(batch)
        done = time.perf_counter() - t0
        gpu_s += time.perf_counter() - g0
        for k, _, _, _ in batch:
            res_lat[k] = done - stream[k][0]
            futs[k] = pool.submit(_crt_job, out[k])
            futs[k].add_done_callback(stamp(k))
        rounds += 1
        i = j
    results = [f.result() for f in futs]
    wall = time.perf_counter() - t0
    stats = {"requests": len(stream), "rounds": rounds, "builds": srv.builds, "plain": srv.plain,
             "resident_gb": srv.used / 1e9, "wall_s": wall, "engine_s": gpu_s,
             "residues_latency": percentiles(res_lat)}
    for tab in srv.chunks.values():
        tab.close()
    if own_pool:
        pool.shutdown()
    return lat, results, stats


def percentiles(lat):
    a = np.sort(np.array(lat))
    if not len(a):
        return {}
    return {"p50_ms": 1e3 * float(np.percentile(a, 50)), "p99_ms": 1e3 * float(np.percentile(a, 99)),
            "max_ms": 1e3 * float(a[-1])}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="serve.py")
    ap.add_argument("--seconds", type=float, default=10)
    ap.add_argument("--rate", type=float, default=200)
    ap.add_argument("--nmin", type=int, default=64)
    ap.add_argument("--nmax", type=int, default=2048)
    ap.add_argument("--budget-gb", type=float, default=150)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--cold", action="store_true", help="start with no resident tables")
    a = ap.parse_args(argv)
    stream = poisson_stream(a.seconds, a.rate, a.nmin, a.nmax, a.seed)
    warm = None if a.cold else [(a.nmax, 4 * a.nmax, d) for d in (2, 3, 4)]
    with cb.Engine(a.device) as eng:
        lat, _, stats = run(stream, eng, a.budget_gb * 1e9, warm=warm)
    print({**percentiles(lat), **stats})
    return 0


if __name__ == "__main__":
    sys.exit(main())
