#!/usr/bin/env python3
"""Continuous-batching query server over resident suffix tables, with its device work overlapped.

A request nbad(n, M, d) is answered as the reference answers it: N_bad modulo the first
need(n, M, d) primes of the fixed list (fast/cuckoo_fast.cu:403-459), recombined by CRT
(crt.py, the fast/post_gmp.py step).  The reference rebuilds a suffix table per prime for every
run.  This server keeps the tables on the GPU across requests (cf_tables_*), per (d, model) in
prime chunks of CHUNK primes, each chunk built to some (n, F) and answering any later request
with n' <= n, M' <= F in O(n'^2) per prime.  A chunk is built, or rebuilt larger, only when a
request needs more than it holds; chunks are admitted under an HBM budget and evicted least
recently used.

Nothing in the loop waits for the device:
* every pass of the loop admits the requests that have arrived (continuous batching), and for
  each chunk that is ready sends the waiting requests' queries as one stream-ordered launch on one
  of a few query streams; results come back through pinned host buffers whose events the loop polls;
* a chunk's build runs on its own stream (cf_tables_build_async) while queries on the ready
  chunks go on; requests that need a chunk still being built wait for it in the queue;
* a request whose tables cannot be resident within the budget takes the plain path: it is rebuilt
  for that request alone (cf_residues) on a worker thread with its own engine, shortest first, its
  launches capped to part of the SMs so resident queries keep running beside it.
The residues of a served request cover whole chunks (the primes beyond its need change nothing:
N_bad is below the product of its own primes), so every CRT is over a prefix of the list whose
length is a multiple of the chunk, and a pool of host processes (crt.PrefixCRT, constants cached
at start) recombines them.  Two latencies are kept per request, from its arrival: residues ready,
and N_bad ready.

    python cuckoo-failure_b200/serve.py [--seconds 10] [--rate 200] [--nmax 2048] [--budget-gb 150] [--seed 1]
"""
import argparse
import concurrent.futures as cf
import heapq
import itertools
import math
import os
import sys
import threading
import time

# Builds, queries and plain rebuilds run on separate streams.  With the driver's default of 8
# hardware work queues, two streams can share one, and a query launched after a plain rebuild's
# queued chunks would wait for all of them; 32 queues keep the streams apart.  It must be set
# before the process creates its CUDA context.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
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


# ---------------------------------------------------------------------------------------------
# Device side
# ---------------------------------------------------------------------------------------------
class GpuBackend:
    """The device side of the server on one GPU: resident tables built on a build stream, queries
    enqueued on query streams into device buffers and copied to pinned host memory, and plain
    rebuilds on a worker thread with its own engine whose launches take at most plain_ctas SMs."""

    def __init__(self, device=0, query_streams=2, plain_ctas=96):
        import torch

        self.torch = torch
        self.device = device
        torch.cuda.set_device(device)
        self.eng = cb.Engine(device)
        self.build_stream = torch.cuda.Stream(device)
        self.qstreams = [torch.cuda.Stream(device) for _ in range(query_streams)]
        self._rr = itertools.cycle(range(query_streams))
        self.plain_ctas = plain_ctas
        self._plain_local = threading.local()
        self.plain_pool = cf.ThreadPoolExecutor(1)

    def build(self, primes, nmax, Fmax, d, model):
        return self.eng.tables_async(primes, nmax, Fmax, d, model, self.build_stream.cuda_stream)

    @staticmethod
    def ready(tab):
        return tab.ready()

    def query(self, tab, queries):
        torch = self.torch
        qs = self.qstreams[next(self._rr)]
        B, J = len(tab.primes), len(queries)
        d_out = torch.empty(B * J, dtype=torch.int64, device=f"cuda:{self.device}")
        host = torch.empty(B * J, dtype=torch.int64, pin_memory=True)
        qs.wait_stream(torch.cuda.current_stream(self.device))  # d_out's allocation
        tab.query_async(queries, d_out.data_ptr(), qs.cuda_stream)
        with torch.cuda.stream(qs):
            host.copy_(d_out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(qs)
        return _GpuTicket(ev, host, d_out, B, J)

    def _plain_engine(self):
        e = getattr(self._plain_local, "eng", None)
        if e is None:
            self.torch.cuda.set_device(self.device)
            e = cb.Engine(self.device)
            e.set_max_ctas(self.plain_ctas)
            self._plain_local.eng = e
        return e

    def _plain_job(self, primes, n, M, d, model):
        """The worker's rebuild of one request: primes in through pinned memory, the launches on the
        worker's own stream, the residues back into pinned memory, and an event polled, so the worker
        never sits inside a blocking CUDA call while the serving loop uses the device."""
        torch = self.torch
        eng = self._plain_engine()
        st = getattr(self._plain_local, "stream", None)
        if st is None:
            st = self._plain_local.stream = torch.cuda.Stream(self.device)
        dev = f"cuda:{self.device}"
        B = len(primes)
        host_p = torch.from_numpy(np.asarray(primes, dtype=np.uint64).view(np.int64)).pin_memory()
        host_o = torch.empty(B, dtype=torch.int64, pin_memory=True)
        with torch.cuda.stream(st):
            d_p = host_p.to(dev, non_blocking=True)
            d_o = torch.empty(B, dtype=torch.int64, device=dev)
        eng.residues_async(d_p.data_ptr(), B, n, d, [(n, M)], d_o.data_ptr(), st.cuda_stream, model=model)
        with torch.cuda.stream(st):
            host_o.copy_(d_o, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        while not ev.query():
            time.sleep(0.002)
        return host_o.numpy().view(np.uint64).copy()

    def plain(self, primes, n, M, d, model):
        """Future of the residues [prime] of (n, M) rebuilt alone, on the worker."""
        return self.plain_pool.submit(self._plain_job, primes, n, M, d, model)

    @staticmethod
    def free(tab):
        tab.close()

    def _close_plain_engine(self):
        e = getattr(self._plain_local, "eng", None)
        if e is not None:
            e.close()
            self._plain_local.eng = None

    def close(self):
        self.plain_pool.submit(self._close_plain_engine).result()  # the worker's engine, in its thread
        self.plain_pool.shutdown(wait=True)
        self.torch.cuda.synchronize(self.device)  # tables freed in stream order are back in the pool
        self.eng.close()


class _GpuTicket:
    def __init__(self, ev, host, d_out, B, J):
        self.ev, self.host, self.d_out, self.B, self.J = ev, host, d_out, B, J

    def done(self):
        return self.ev.query()

    def result(self):
        self.ev.synchronize()
        self.d_out = None
        return self.host.numpy().view(np.uint64).reshape(self.B, self.J)


# ---------------------------------------------------------------------------------------------
# The scheduling loop
# ---------------------------------------------------------------------------------------------
class _Chunk:
    def __init__(self, key, tab, nmax, Fmax, nbytes):
        self.key, self.tab, self.nmax, self.Fmax, self.bytes = key, tab, nmax, Fmax, nbytes
        self.ready = False
        self.inflight = 0  # query launches not yet returned

    def covers(self, n, M):
        return self.nmax >= n and self.Fmax >= M


class _Req:
    __slots__ = ("rid", "n", "M", "d", "chunks", "got", "plain", "sent")

    def __init__(self, rid, n, M, d, nchunks):
        self.rid, self.n, self.M, self.d = rid, n, M, d
        self.chunks = list(range(nchunks))
        self.got = {}  # chunk -> residues of its primes
        self.sent = set()  # chunks whose query is in flight
        self.plain = False


class Server:
    """Request scheduling over a backend (GpuBackend, or a stand-in in tests).

    submit() queues a request; pump() runs one pass of the loop and returns the requests whose
    residues are complete as [(rid, residues)], residues covering at least need(n, M, d) primes."""

    def __init__(self, backend, budget_bytes, model=cb.MODEL_SUBSET, n_cap=16384, chunk=CHUNK, bytes_fn=None,
                 plain_nmax=None, resident_nmax=None):
        self.be, self.budget, self.model, self.n_cap, self.chunk = backend, budget_bytes, model, n_cap, chunk
        self.plain_nmax = plain_nmax  # plain requests above this n are refused (None: no bound)
        # requests above this n take the plain path even when their tables would fit, so they never
        # evict the tables that serve the requests below it (None: any that fit are made resident)
        self.resident_nmax = resident_nmax
        self.refused = []
        self.bytes_fn = bytes_fn or cb.tables_bytes
        self.chunks = OrderedDict()  # (d, chunk index) -> _Chunk, LRU order (the chunk queries use)
        self.building = {}           # (d, chunk index) -> _Chunk being built to replace or add
        self.retired = []            # replaced chunks, freed once no query on them is in flight
        self.used = 0
        self.pending = OrderedDict()  # rid -> _Req waiting for tables or queries
        self.tickets = []            # (ticket, chunk, [(req, query column)])
        self.plain_futs = []         # (future, req)
        self.plain_heap = []         # (work estimate, rid) waiting for the worker
        self.plain_busy = 0
        self.builds = self.plain = self.launches = 0

    # -- admission -----------------------------------------------------------------------------
    def submit(self, rid, n, M, d):
        k = cb.need(n, M, d, self.model)
        r = _Req(rid, n, M, d, (k + self.chunk - 1) // self.chunk)
        if not self._can_hold(r) or (self.resident_nmax is not None and n > self.resident_nmax):
            if self.plain_nmax is not None and n > self.plain_nmax:
                self.refused.append(rid)  # a rebuild this large cannot be interrupted: not taken
                return
            r.plain = True
            heapq.heappush(self.plain_heap, (k * float(n) ** 2, rid))
        self.pending[rid] = r

    def _size(self, d, c, n, M):
        old = self.chunks.get((d, c))
        n2 = min(self.n_cap, max(grow(n), old.nmax if old else 0))
        F2 = max(grow(M), old.Fmax if old else 0, n2)
        return n2, F2, self.chunk * self.bytes_fn(n2, F2)

    def _can_hold(self, r):
        """Whether the request's chunks at its size could be resident together within the budget."""
        tot = sum(self._size(r.d, c, r.n, r.M)[2] for c in r.chunks)
        return tot <= self.budget

    # -- residency -------------------------------------------------------------------------------
    def _evict_for(self, need_bytes, keep):
        for key in list(self.chunks):
            if self.used + need_bytes <= self.budget:
                break
            ch = self.chunks[key]
            if key in keep or ch.inflight or key in self.building:
                continue
            del self.chunks[key]
            self.used -= ch.bytes
            self.be.free(ch.tab)
        return self.used + need_bytes <= self.budget

    def _start_build(self, d, c, n, M, keep):
        n2, F2, nbytes = self._size(d, c, n, M)
        if not self._evict_for(nbytes, keep):
            return False
        primes = cb.prime_range(c * self.chunk, self.chunk)
        tab = self.be.build(primes, n2, F2, d, self.model)
        self.building[(d, c)] = _Chunk((d, c), tab, n2, F2, nbytes)
        self.used += nbytes
        self.builds += 1
        return True

    def _poll_builds(self):
        for key, ch in list(self.building.items()):
            if not self.be.ready(ch.tab):
                continue
            del self.building[key]
            ch.ready = True
            old = self.chunks.pop(key, None)
            if old is not None:  # replaced by a larger table: freed once its queries are back
                self.retired.append(old)
            self.chunks[key] = ch

    def _free_retired(self):
        keep = []
        for ch in self.retired:
            if ch.inflight:
                keep.append(ch)
            else:
                self.used -= ch.bytes
                self.be.free(ch.tab)
        self.retired = keep

    # -- one pass of the loop --------------------------------------------------------------------
    def pump(self):
        done = []
        # results that came back
        still = []
        for tk, ch, items in self.tickets:
            if not tk.done():
                still.append((tk, ch, items))
                continue
            out = tk.result()
            ch.inflight -= 1
            for req, jj in items:
                req.got[ch.key[1]] = out[:, jj]
                req.sent.discard(ch.key[1])
                if len(req.got) == len(req.chunks):
                    done.append((req.rid, [int(x) for c in req.chunks for x in req.got[c]]))
                    del self.pending[req.rid]
        self.tickets = still
        still = []
        for fut, req in self.plain_futs:
            if fut.done():
                done.append((req.rid, [int(x) for x in fut.result()]))
                del self.pending[req.rid]
                self.plain_busy -= 1
            else:
                still.append((fut, req))
        self.plain_futs = still
        self._poll_builds()
        # plain requests: one at a time on the worker, the least work first
        while self.plain_heap and self.plain_busy == 0:
            _, rid = heapq.heappop(self.plain_heap)
            req = self.pending[rid]
            primes = cb.prime_range(0, cb.need(req.n, req.M, req.d, self.model))
            self.plain_futs.append((self.be.plain(primes, req.n, req.M, req.d, self.model), req))
            self.plain_busy += 1
            self.plain += 1
        # Resident requests, oldest first.  A request is provisioned when every chunk it needs is
        # resident or being built at a size that covers it; its missing builds start together or
        # not at all, evicting only chunks no provisioned request holds, and a request that does
        # not fit stops the builds of the requests behind it (so the oldest always gets through
        # once the ones ahead of it are answered, and no two requests hold parts of each other's
        # room).  Per ready chunk, one query launch goes out for every request waiting on it.
        wanted = {}
        keep = set()
        blocked = False
        for req in self.pending.values():
            if req.plain:
                continue
            missing = []
            for c in req.chunks:
                key = (req.d, c)
                ch, b = self.chunks.get(key), self.building.get(key)
                if not (ch is not None and ch.covers(req.n, req.M)) and not (b is not None and b.covers(req.n, req.M)):
                    missing.append(c)
            if missing:
                if blocked or any((req.d, c) in self.building for c in missing):
                    blocked = True  # a build of too small a size is still running: wait for it
                else:
                    # a chunk resident at too small a size is replaced: its room counts as free once
                    # no query on it is in flight and no request ahead holds it
                    mine = keep | {(req.d, c) for c in req.chunks if c not in missing}
                    need_bytes = sum(self._size(req.d, c, req.n, req.M)[2] for c in missing)
                    if self._evict_for(need_bytes, mine):
                        for c in missing:
                            self._start_build(req.d, c, req.n, req.M, mine)
                        missing = []
                    else:
                        blocked = True
            if not missing:
                keep |= {(req.d, c) for c in req.chunks}
            for c in req.chunks:
                if c in req.got or c in req.sent:
                    continue
                key = (req.d, c)
                ch = self.chunks.get(key)
                if ch is not None and ch.ready and ch.covers(req.n, req.M):
                    wanted.setdefault(key, []).append(req)
        for key, reqs in wanted.items():
            ch = self.chunks[key]
            self.chunks.move_to_end(key)
            tk = self.be.query(ch.tab, [(r.n, r.M) for r in reqs])
            ch.inflight += 1
            self.launches += 1
            for r in reqs:
                r.sent.add(key[1])
            self.tickets.append((tk, ch, [(r, jj) for jj, r in enumerate(reqs)]))
        self._free_retired()
        return done

    def idle(self):
        return not self.pending

    def close(self):
        for ch in list(self.chunks.values()) + list(self.building.values()) + self.retired:
            self.be.free(ch.tab)
        self.chunks.clear()
        self.building.clear()
        self.retired = []


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
    import multiprocessing as mp

    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    kmax = ((max_primes + chunk - 1) // chunk) * chunk
    primes = [int(p) for p in cb.prime_range(0, kmax)]
    warm = list(range(chunk, kmax + 1, chunk))
    pool = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                  initializer=_crt_init, initargs=(primes, warm))
    list(pool.map(time.sleep, [0.05] * (2 * workers)))  # every worker started and warm
    return pool


def run(stream, backend, budget_bytes, model=cb.MODEL_SUBSET, warm=None, chunk=CHUNK, pool=None, drain_s=None,
        bytes_fn=None, plain_nmax=None, resident_nmax=None):
    """Serve a timed stream [(arrival_s, n, M, d)] in real time.  `warm`, if given, is a list of
    (n, M, d) whose chunks are built (and waited for) before the clock starts.  After the last
    arrival the loop runs until every request is answered, or for at most drain_s seconds.
    plain_nmax, if given, refuses plain-path requests above that n (counted, never answered);
    resident_nmax, if given, sends every request above that n to the plain path.
    Returns (latencies_s, results, stats): latency to N_bad and N_bad per request (None when not
    answered in time), and counters including the latency to residues."""
    srv = Server(backend, budget_bytes, model, chunk=chunk, bytes_fn=bytes_fn, plain_nmax=plain_nmax,
                 resident_nmax=resident_nmax)
    for n, M, d in warm or []:
        for c in range((cb.need(n, M, d, model) + chunk - 1) // chunk):
            srv._start_build(d, c, n, M, set())
    while srv.building:
        srv._poll_builds()
        time.sleep(0.002)
    warm_builds = srv.builds
    own_pool = pool is None
    if own_pool:
        kmax = max([cb.need(n, M, d, model) for _, n, M, d in stream] + [1])
        pool = crt_pool(kmax, chunk)
    futs = [None] * len(stream)
    lat, res_lat = [None] * len(stream), [None] * len(stream)
    t0 = time.perf_counter()
    i = 0
    last = stream[-1][0] if stream else 0.0

    def stamp(k):
        def cb_(_f):
            lat[k] = time.perf_counter() - t0 - stream[k][0]
        return cb_

    passes = 0
    while True:
        now = time.perf_counter() - t0
        while i < len(stream) and stream[i][0] <= now:
            _, n, M, d = stream[i]
            srv.submit(i, n, M, d)
            i += 1
        for rid, residues in srv.pump():
            res_lat[rid] = time.perf_counter() - t0 - stream[rid][0]
            futs[rid] = pool.submit(_crt_job, residues)
            futs[rid].add_done_callback(stamp(rid))
        passes += 1
        if i >= len(stream) and (srv.idle() or (drain_s is not None and now > last + drain_s)):
            break
        if srv.idle() and i < len(stream):
            time.sleep(max(0.0, min(stream[i][0] - now, 0.002)))
        else:
            time.sleep(0.0002)
    wall = time.perf_counter() - t0
    results = [f.result() if f is not None else None for f in futs]
    unanswered = sum(1 for r in res_lat if r is None)
    stats = {"requests": len(stream), "answered": len(stream) - unanswered, "unanswered": unanswered,
             "refused": len(srv.refused), "loop_passes": passes, "query_launches": srv.launches,
             "builds": srv.builds - warm_builds,
             "warm_builds": warm_builds, "plain": srv.plain, "resident_gb": srv.used / 1e9, "wall_s": wall,
             "residues_latency": percentiles([x for x in res_lat if x is not None])}
    srv.close()
    if own_pool:
        pool.shutdown()
    return lat, results, stats


def percentiles(lat):
    a = np.sort(np.array([x for x in lat if x is not None], dtype=float))
    if not len(a):
        return {}
    return {"p50_ms": 1e3 * float(np.percentile(a, 50)), "p99_ms": 1e3 * float(np.percentile(a, 99)),
            "max_ms": 1e3 * float(a[-1]), "count": int(len(a))}


def bucketed(stream, lat, edges=(512, 2048, 8192, 16384)):
    """Latency percentiles per n bucket: {"n<=512": {...}, ...}, with the unanswered count."""
    out, lo = {}, 0
    for e in edges:
        ks = [k for k, (_, n, _, _) in enumerate(stream) if lo < n <= e]
        got = [lat[k] for k in ks if lat[k] is not None]
        out[f"{lo + 1}..{e}"] = {**percentiles(got), "requests": len(ks), "unanswered": len(ks) - len(got)}
        lo = e
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="serve.py")
    ap.add_argument("--seconds", type=float, default=10)
    ap.add_argument("--rate", type=float, default=200)
    ap.add_argument("--nmin", type=int, default=64)
    ap.add_argument("--nmax", type=int, default=2048)
    ap.add_argument("--budget-gb", type=float, default=150)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--drain-s", type=float, default=None)
    ap.add_argument("--cold", action="store_true", help="start with no resident tables")
    a = ap.parse_args(argv)
    stream = poisson_stream(a.seconds, a.rate, a.nmin, a.nmax, a.seed)
    warm = None if a.cold else [(min(a.nmax, 2048), 4 * min(a.nmax, 2048), d) for d in (2, 3, 4)]
    be = GpuBackend(a.device)
    lat, _, stats = run(stream, be, a.budget_gb * 1e9, warm=warm, drain_s=a.drain_s)
    be.close()
    print({**percentiles(lat), **stats, "buckets": bucketed(stream, lat)})
    return 0


if __name__ == "__main__":
    sys.exit(main())
