#!/usr/bin/env python3
"""Throughput of the one-table suffix-table engine: prime-residues/s at n=16384, M=32768, d=3.

One step = one batch of B primes through the hot path: per-prime tables, the n-1 suffix-table
steps (two 1/t convolutions each), the nbad(n, M) query and the Horner finish, for every prime.
The device-timed step replays the batch captured once as a CUDA graph (cf_batch_graph_*); the
e2e figure goes through cf_residues with host buffers.
A prime-residue is one (d, prime) table built to n plus the residue of its query.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) each rank takes its own disjoint prime range (weak scaling, no collective
on the data path); the time is the max over ranks.  `--impl reference` times the reference's own
CPU build (oracle/_ref/cuckoo_fast_ifma, or _cpu without AVX-512 IFMA) in one process per host
core on disjoint primes, the reference's documented way to split a run.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

# the serving run overlaps streams (builds, queries, plain rebuilds): keep them on separate hardware
# work queues; read when the CUDA context is created, so it is set before anything touches the GPU
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuckoo-failure_b200")
sys.path.insert(0, PKG)

METRIC = "prime-residues/s, n=16384 d=3 NTT suffix build; served-query p50/p99 latency"
UNIT = "prime-residues/s"
K_OPS_PER_MM = 20  # INT32 multiply ops per 64-bit modular multiplication (fixed accounting model)
# DRAM bytes (read + write) per prime of the engine kernel, from an ncu capture of this bench at 2
# primes per launch (profiles/k_suffix_n16384_b2_sections.md), keyed by (n, M, d, prime bits); the
# bench scales it by the primes per launch
MEASURED_TRAFFIC_PER_PRIME = {(16384, 32768, 3, 50): (4.138317e9 + 4.254311e9) / 2}
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def algorithmic_mm(n):
    """Modular multiplications per prime-residue (one table to n plus one query): two convolutions
    per step of L (lg + 1) each, the stage pre/post products (about 6.5 n^2) and the query (1.5 n^2)."""
    L = 16
    while L < n:
        L *= 2
    lg = L.bit_length() - 1
    return 2 * (n - 1) * L * (lg + 1) + 8 * n * n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.thread.join(timeout=2)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def hbm_peak():
    """Copy bandwidth of this pool's B200s (GB/s): the measured-peaks file beside this script, else
    the earlier measurement on the same pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_binary():
    ifma = os.path.join(REF_DIR, "cuckoo_fast_ifma")
    has_ifma = "avx512ifma" in open("/proc/cpuinfo").read()
    if has_ifma and os.path.exists(ifma):
        return ifma, "AVX-512 IFMA build (make fast-ifma)"
    return os.path.join(REF_DIR, "cuckoo_fast_cpu"), "scalar host build (make fast)"


def run_reference_wave(binary, n, M, d, first, procs):
    """One process per core, each one prime of the fixed list (disjoint FIRST COUNT ranges).
    Returns (seconds, output lines)."""
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(f"{n} {M}\n")
        qpath = f.name
    t0 = time.perf_counter()
    ps = [subprocess.Popen([binary, str(d), qpath, str(first + k), "1"], stdout=subprocess.PIPE,
                           stderr=subprocess.DEVNULL, text=True) for k in range(procs)]
    outs = [p.communicate()[0] for p in ps]
    dt = time.perf_counter() - t0
    os.unlink(qpath)
    if any(p.returncode for p in ps):
        raise RuntimeError("reference binary failed")
    return dt, [ln for o in outs for ln in o.splitlines()]


def reference_gpu(n, M, d, primes=64, timeout_s=900):
    """The reference's CUDA build (fast/cuckoo_fast.cu compiled by its own `fast-gpu` recipe, with an
    sm_100a target: oracle/Makefile.ref) on this GPU: primes 0 .. primes-1 in one run, its default
    batch (at most 64 primes, fast/cuckoo_fast.cu:743-747).  The rate is over the run's own clock
    up to its queries done (setup, uploads, the step loop, k_query, download, Horner finish), which
    leaves out only process start and CUDA context creation; its residues for primes 0 and 1 are
    checked against the reference host build's."""
    import re

    binary = os.path.join(REF_DIR, "cuckoo_fast_gpu")
    if not os.path.exists(binary):
        return None
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(f"{n} {M}\n")
        qpath = f.name
    t0 = time.perf_counter()
    r = subprocess.run([binary, str(d), qpath, "0", str(primes)], capture_output=True, text=True, timeout=timeout_s)
    wall = time.perf_counter() - t0
    os.unlink(qpath)
    if r.returncode:
        return {"unavailable": f"exit {r.returncode}: {r.stderr.strip()[-200:]}"}
    m = re.search(r"build done at ([0-9.]+) s, queries at ([0-9.]+) s", r.stderr)
    got = {int(t[0]): int(t[4]) for t in (ln.split() for ln in r.stdout.splitlines()) if len(t) == 5}
    for i, want in golden_check(n, M, d).items():
        assert got.get(i) == want, f"reference CUDA build: residue mismatch at prime {i}"
    done = float(m.group(2)) if m else wall
    return {"value": primes / done, "unit": UNIT, "primes": primes, "build_done_s": float(m.group(1)) if m else None,
            "queries_done_s": done, "wall_s": wall,
            "what": "the reference's CUDA build on this GPU, one run over primes 0..%d at n=%d, M=%d, d=%d" % (primes - 1, n, M, d)}


def cpu_baseline(n, M, d):
    binary, kind = reference_binary()
    P = host_cores()
    dt, lines = run_reference_wave(binary, n, M, d, 0, P)
    return {"value": P / dt, "unit": UNIT, "cores": P, "kind": "reference",
            "sample": f"{P} processes x 1 prime (primes 0..{P - 1}) of n={n}, M={M}, d={d} with the reference's "
                      f"{kind}, {dt:.1f} s wall"}


def golden_check(n, M, d, bits=50):
    """Known residues of the reference host build (tests/golden): primes 0 and 1, and 0 .. 15 at
    the headline size."""
    out = {}
    for suffix in ("", "_first16"):
        path = os.path.join(ROOT, "tests", "golden", f"fast{'62' if bits == 62 else ''}_n{n}_d{d}{suffix}.txt")
        if not os.path.exists(path):
            continue
        with open(path) as f:
            for ln in f:
                t = ln.split()
                if len(t) == 5 and not ln.startswith("#") and int(t[2]) == n and int(t[3]) == M:
                    out[int(t[0])] = int(t[4])
    return out


def serving_run(device, seconds, rate=200.0, budget_gb=150.0, full_seconds=2.0, drain_s=20.0, plain_nmax=4096):
    """Served-query latency through serve.py's loop (resident tables, builds on their own stream,
    queries overlapped on query streams, plain rebuilds on a worker), seeded Poisson streams at
    `rate` per second with M = n U[1.5, 4] and d in {2, 3, 4}:
    * the resident range: n log-uniform in [64, 2048] for `seconds`, tables for (2048, 8192, d)
      built before the clock (they fit the budget for every d);
    * the full range the workload states, n log-uniform in [64, 16384], for `full_seconds` with
      the same warm tables; requests above the resident range (n > 2048, whose tables would evict
      the ones that serve the rest) take the plain path one at a time,
      least work first (up to n = plain_nmax; a rebuild cannot be interrupted, so larger ones are
      refused), and the loop stops `drain_s` after the last arrival: what is not answered by then
      is counted per n bucket.
    Latencies from arrival to residues ready and to exact N_bad (after the host CRT pool), per n
    bucket.  Beside them, the plain form: one request of each size class rebuilt alone."""
    import numpy as np

    import cuckoo_b200 as cb
    import serve

    warm = [(2048, 8192, dd) for dd in (2, 3, 4)]
    out = {}
    be = serve.GpuBackend(device)
    try:
        for key, secs, n_hi, drain in (("resident_range", seconds, 2048, None), ("full_range", full_seconds, 16384, drain_s)):
            stream = serve.poisson_stream(secs, rate, 64, n_hi, seed=20261203)
            kmax = max(cb.need(n, M, dd) for _, n, M, dd in stream)
            pool = serve.crt_pool(kmax)
            lat, _, st = serve.run(stream, be, budget_gb * 1e9, warm=warm, pool=pool, drain_s=drain,
                                   plain_nmax=plain_nmax if drain is not None else None, resident_nmax=2048)
            pool.shutdown()
            rl = st["residues_latency"]
            nb = serve.percentiles(lat)
            out[key] = {
                "workload": f"Poisson {rate:g} req/s for {secs:g} s, n log-uniform [64, {n_hi}], M/n U[1.5, 4], "
                            f"d in {{2,3,4}}; {budget_gb:g} GB table budget; tables for n <= 2048 built before the clock",
                "p50_ms": rl.get("p50_ms"), "p99_ms": rl.get("p99_ms"), "latency_to": "residues ready",
                "nbad_p50_ms": nb.get("p50_ms"), "nbad_p99_ms": nb.get("p99_ms"),
                "buckets_nbad": serve.bucketed(stream, lat),
                "requests": st["requests"], "answered": st["answered"], "plain_path_requests": st["plain"],
                "refused_plain_above_n": plain_nmax if drain is not None else None, "refused": st["refused"],
                "builds_during_stream": st["builds"], "query_launches": st["query_launches"],
                "requests_per_s": st["answered"] / st["wall_s"], "resident_gb": st["resident_gb"], "wall_s": st["wall_s"]}
        with cb.Engine(device) as eng:  # the plain form: one request rebuilt alone, per size class
            plain = {}
            for n in (256, 1024, 4096):
                M, dd = 3 * n, 3
                ps = cb.prime_range(0, cb.need(n, M, dd))
                eng.residues(ps[:2], n, dd, [(n, M)])
                t0 = time.perf_counter()
                eng.residues(ps, n, dd, [(n, M)])
                plain[f"n={n},M={M},d={dd}"] = {"primes": len(ps), "ms": 1e3 * (time.perf_counter() - t0)}
        out["plain_rebuild"] = plain
        out["note"] = ("a table at n = 16384 is 1.07 GB per prime and a d = 3 request there needs 14184 primes (15 TB): "
                       "n above ~2048 cannot stay resident for d = 2..4 within the budget, and one such request alone "
                       "takes the plain path's full-GPU time (about need / rate: minutes at n = 16384); the full-range "
                       "stream offers far more plain work than the GPU can do, so its upper buckets stay unanswered")
    finally:
        be.close()
    return out


def timed_replays(launch, stream, reps):
    """Device time (ms) of `reps` back-to-back calls of launch(stream_ptr) on `stream`, after one warm-up."""
    import torch

    launch(stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def uneven_run(eng, stride, per_instance_count=32, seed=None):
    """The uneven-batch workload (512 instances: n log-uniform in [256, 16384], M = n U{2, 3, 4},
    d in {2, 3, 4}, seed-fixed), every instance modulo its own need(n, M, d) primes, on the prime
    indices that are multiples of `stride` (a sample whose tables follow the whole run's mix),
    as one graph of work-queue launches.  Beside it the plain form, each instance alone (one
    cf_residues call, a launch per chunk of primes, per instance), measured like for like against
    the graph on the first per_instance_count instances and the same primes; and a work model of
    the whole run (sum over tables of (n - 1) L (lg L + 1), in tables of n = 16384) for both forms."""
    import cuckoo_b200 as cb
    import uneven

    insts = uneven.instances(512, seed=seed or uneven.CONFIG4_SEED)
    needs = [cb.need(n, M, d) for n, M, d in insts]
    planned = [len(range(0, k, stride)) for k in needs]

    def graph_time(instances):
        import torch

        stream = torch.cuda.Stream()
        with eng.uneven(instances, stride=stride) as u:
            ms = timed_replays(u.launch, stream, 1)
            return ms, u.results(stream.cuda_stream), u.tables(), u.launches()

    ms, res, tables, launches = graph_time(insts)
    sub = insts[:per_instance_count]
    sub_ms, sub_res, sub_tables, _ = graph_time(sub)
    t0 = time.perf_counter()
    alone = uneven.per_instance(eng, sub, cb.prime_range, cb.need, stride=stride)
    plain_s = time.perf_counter() - t0
    for k in range(len(sub)):  # the same residues every way
        assert [int(x) for x in res[k][::stride]] == [int(x) for x in sub_res[k][::stride]] == alone[k][::stride], \
            f"uneven instance {k} differs"

    def cost(n):
        L = cb.transform_length(n)
        return (n - 1) * L * L.bit_length()

    full = cb.uneven_describe(insts)
    c16 = cost(16384)
    queue_equiv = sum(cost(t[3]) for t in full) / c16
    plain_equiv = sum(k * cost(n) for (n, _, _), k in zip(insts, needs)) / c16
    return {"workload": "512 instances, n log-uniform [256, 16384], M = n U{2,3,4}, d U{2,3,4}, "
                        f"seed {uneven.CONFIG4_SEED}; prime indices i = 0 mod {stride} of each instance's need",
            "graph": {"tables": tables, "launches_per_graph": launches, "ms": ms, "tables_per_s": tables / (ms * 1e-3),
                      "instance_residues": sum(planned), "instance_residues_per_s": sum(planned) / (ms * 1e-3),
                      "tables_full_run": len(full), "full_run_s_est": len(full) / (tables / (ms * 1e-3))},
            "like_for_like": {"instances": per_instance_count, "instance_residues": sum(planned[:per_instance_count]),
                              "graph_ms": sub_ms, "graph_tables": sub_tables, "per_instance_s": plain_s,
                              "speedup": plain_s / (sub_ms * 1e-3),
                              "what": "the first instances, same primes: one graph against one cf_residues call per instance"},
            "work_model": {"graph_tables_of_n16384": queue_equiv, "per_instance_tables_of_n16384": plain_equiv,
                           "ratio": plain_equiv / queue_equiv,
                           "what": "whole run: one table per (d, prime) at its largest n, against one per (instance, prime)"}}


def config2_run(device, n=4096, M=8192, d=3, waves=4, reps=3):
    """The batch-scale configuration (n = 4096, M = 8192, d = 3): the engine's geometries for
    transform length 2^12 timed by the autotuner on `waves` x #SMs primes, then the chosen and the
    default geometry each timed as one graph-captured launch of that batch, the residues of primes
    0..3 checked against the reference's."""
    import numpy as np
    import torch

    import cuckoo_b200 as cb

    sms = torch.cuda.get_device_properties(device).multi_processor_count
    B = waves * sms
    out = {"workload": f"n={n}, M={M}, d={d}, {B} primes per launch"}
    stream = torch.cuda.Stream()
    with cb.Engine(device) as eng:
        rec = eng.autotune(n, M, d, B)
        out["autotune"] = rec
        primes = cb.prime_range(0, B)
        d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
        d_out = torch.empty(B, dtype=torch.int64, device="cuda")
        gold = golden_check(n, M, d)
        for label, k in (("default", 0), ("tuned", rec["chosen"])):
            eng.tune_set(rec["lg"], k)
            g = eng.batch_graph(d_primes.data_ptr(), B, n, d, [(n, M)], d_out.data_ptr())
            ms = timed_replays(g.launch, stream, reps)
            g.status(stream.cuda_stream)
            g.close()
            got = d_out.cpu().numpy().view(np.uint64)
            for i, r in gold.items():
                assert int(got[i]) == r, f"config 2 ({label}): residue mismatch at prime {i}"
            out[label] = {"geometry": rec["variants"][k], "value": B / (ms * 1e-3), "unit": UNIT, "ms_per_launch": ms,
                          "frac_top": B * algorithmic_mm(n) * K_OPS_PER_MM / (ms * 1e-3) / 1e12}
    return out


def sweep_run(eng, n, M, B, reps=2):
    """Config-3 sweep at n = 16384, M = 2n: d = 2 and 4 (subset model), the replacement model at
    d = 3, and d = 3 on the list of primes below 2^62 (the reference's -DFP_RB=64 build); one
    graph-captured 148-prime launch per step, the residues checked where the reference has them."""
    import numpy as np
    import torch

    import cuckoo_b200 as cb

    out = {}
    stream = torch.cuda.Stream()
    for d, model, bits in ((2, cb.MODEL_SUBSET, 50), (4, cb.MODEL_SUBSET, 50), (3, cb.MODEL_REPLACEMENT, 50),
                           (3, cb.MODEL_SUBSET, 62)):
        primes = cb.prime_range(0, B, bits=bits)
        assert cb.lib().cf_engine_set_prime_bits(eng._h, bits) == 0  # the graph does not read its primes
        d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
        d_out = torch.empty(B, dtype=torch.int64, device="cuda")
        g = eng.batch_graph(d_primes.data_ptr(), B, n, d, [(n, M)], d_out.data_ptr(), model=model)
        ms = timed_replays(g.launch, stream, reps)
        g.status(stream.cuda_stream)
        g.close()
        got = d_out.cpu().numpy().view(np.uint64)
        if model == cb.MODEL_SUBSET:
            for i, r in golden_check(n, M, d, bits).items():
                assert int(got[i]) == r, f"d={d}, {bits}-bit primes: residue mismatch at prime {i}"
        key = f"d{d}" + ("_replacement" if model else "") + ("_62bit" if bits == 62 else "")
        out[key] = {"value": B / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": reps,
                    "primes_needed": cb.need(n, M, d, model, bits=bits),
                    "frac": B * algorithmic_mm(n) * K_OPS_PER_MM / (ms * 1e-3) / 1e12}
    assert cb.lib().cf_engine_set_prime_bits(eng._h, 50) == 0
    return out


def large_run(device, sizes=((32768, 65536), (65536, 131072)), d=3, reps=1):
    """Tables above n = 16384 (one prime per thread-block cluster): per size, as many primes as fit
    the device (one fewer), rounded down to whole waves of resident clusters, one graph-captured
    launch timed after a warm-up, and one prime alone; residues of primes 0 and 1 checked against the reference host build's.  Beside it
    the reference's only published timing, at n = 65536 on an H100 (fast/README.md:80-86)."""
    import numpy as np
    import torch

    import cuckoo_b200 as cb

    out = {}
    stream = torch.cuda.Stream()
    for n, M in sizes:
        with cb.Engine(device) as eng:
            fit, wave = max(1, eng.max_batch(n, M, 1) - 1), eng.resident_primes(n, M, 1)
            B = fit - fit % wave if wave and fit > wave else fit  # whole waves of resident clusters
            primes = cb.prime_range(0, B)
            d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
            d_out = torch.empty(B, dtype=torch.int64, device="cuda")
            g = eng.batch_graph(d_primes.data_ptr(), B, n, d, [(n, M)], d_out.data_ptr())
            ms = timed_replays(g.launch, stream, reps)
            g.status(stream.cuda_stream)
            g.close()
            got = d_out.cpu().numpy().view(np.uint64)
            for i, r in golden_check(n, M, d).items():
                assert int(got[i]) == r, f"n={n}: residue mismatch at prime {i}"
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            eng.residues_async(d_primes.data_ptr(), 1, n, d, [(n, M)], d_out.data_ptr(), stream.cuda_stream)
            q1.record(stream)
            torch.cuda.synchronize()
            one = q0.elapsed_time(q1)
        out[f"n{n}"] = {"value": B / (ms * 1e-3), "unit": UNIT, "primes_per_launch": B, "ms_per_launch": ms,
                        "one_prime_alone_s": one * 1e-3, "workload": f"n={n}, M={M}, d={d}, one query, 50-bit primes",
                        "checked": "residues of primes 0 and 1 equal the reference host build's"}
    # the reference's published case: n = 65536 with 126 queries (the seeded set of the fixture)
    path = os.path.join(ROOT, "tests", "golden", "fast_n65536_d3_J126.txt")
    if os.path.exists(path):
        with open(path) as f:
            head = f.readline()
            want = {(int(t[2]), int(t[3])): int(t[4]) for t in (ln.split() for ln in f) if len(t) == 5 and t[0] == "0"}
        qs = [tuple(int(x) for x in tok.split(",")) for tok in head.split("queries=")[1].split(" first=")[0].split()]
        n, M = 65536, max(m for _, m in qs)
        with cb.Engine(device) as eng:
            fit, wave = max(1, eng.max_batch(n, M, len(qs)) - 1), eng.resident_primes(n, M, len(qs))
            B = fit - fit % wave if wave and fit > wave else fit
            primes = cb.prime_range(0, B)
            d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
            d_out = torch.empty(B * len(qs), dtype=torch.int64, device="cuda")
            g = eng.batch_graph(d_primes.data_ptr(), B, n, d, qs, d_out.data_ptr())
            ms = timed_replays(g.launch, stream, reps)
            g.status(stream.cuda_stream)
            g.close()
            got = d_out.cpu().numpy().view(np.uint64)[:len(qs)]
            assert all(int(r) == want[q] for q, r in zip(qs, got)), "n=65536, 126 queries: residue mismatch at prime 0"
        out["n65536_J126"] = {"value": B / (ms * 1e-3), "unit": UNIT, "primes_per_launch": B, "ms_per_launch": ms,
                              "queries": len(qs), "s_per_prime_at_this_rate": ms * 1e-3 / B,
                              "workload": "n=65536, d=3, 126 queries (n from 2000 to 65536, M = n U[1.5, 4], seeded)",
                              "checked": "all 126 residues of prime 0 equal the reference host build's"}
    out["reference_published"] = ("fast/README.md:80-86: n = 65536, one prime, 126 queries, CUDA batch 2 on an H100: "
                                  "table build 3.5 s per prime, queries 0.75 s (current version)")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--M", type=int, default=32768)
    ap.add_argument("--d", type=int, default=3)
    ap.add_argument("--batch", type=int, default=0, help="primes per step per GPU (default: one wave)")
    ap.add_argument("--prime-bits", type=int, default=50, choices=[50, 62],
                    help="prime list: below 2^50 (default) or below 2^62 (the reference's -DFP_RB=64 build)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-query latency run")
    ap.add_argument("--no-plain-form", action="store_true", help="skip the one-prime-per-launch timing")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-full-seconds", type=float, default=2.0,
                    help="length of the full-range (n up to 16384) serving stream")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch (512 instances) run")
    ap.add_argument("--uneven-stride", type=int, default=97)
    ap.add_argument("--no-sweep", action="store_true", help="skip d = 2, 4 and the replacement model")
    ap.add_argument("--no-config2", action="store_true", help="skip the n = 4096 (autotuned) run")
    ap.add_argument("--no-large", action="store_true", help="skip the tables above n = 16384 (n = 32768, 65536)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="--impl reference: skip the reference's CUDA build (timed beside its host build)")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="DRAM bytes per launch of the main kernel from an ncu capture (roofline.traffic)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    n, M, d = a.n, a.M, a.d
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    workload = f"one-table suffix build + nbad query, n={n}, M={M}, d={d}, {a.prime_bits}-bit primes of the fixed list"

    if a.impl == "reference":
        if rank != 0:
            return 0
        binary, kind = reference_binary()
        if not os.path.exists(binary):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (run make -f oracle/Makefile.ref)"}))
            return 0
        P = host_cores()
        times = []
        for s in range(a.warmup + a.steps):
            dt, _ = run_reference_wave(binary, n, M, d, s * P, P)
            if s >= a.warmup:
                times.append(dt)
        tot = sum(times)
        v = P * a.steps / tot
        rgpu = reference_gpu(n, M, d) if not a.no_reference_gpu else None
        print(json.dumps({
            "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": workload, "batch_primes_per_step": P, "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": P, "kind": "reference",
                             "sample": f"each step {P} processes x 1 prime with the reference's {kind}"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu": rgpu}))
        return 0

    import ctypes

    import numpy as np
    import torch

    import cuckoo_b200 as cb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    eng = cb.Engine(local)
    queries = [(n, M)]
    J = 1
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    # one wave, one prime below what fits now: what the launch sees must still hold the whole batch
    B = a.batch or max(1, min(eng.max_batch(n, M, J) - 1, sms))
    primes = cb.prime_range(rank * B, B, bits=a.prime_bits)
    if a.prime_bits != 50:
        lib_rc = cb.lib().cf_engine_set_prime_bits(eng._h, a.prime_bits)
        assert lib_rc == 0
    stream = torch.cuda.Stream()  # a dedicated stream: the events below are recorded on it
    d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
    d_out = torch.empty(B * J, dtype=torch.int64, device="cuda")

    # the batch as one CUDA graph (error-word reset + the persistent launch), replayed every step
    graph = eng.batch_graph(d_primes.data_ptr(), B, n, d, queries, d_out.data_ptr())

    def step():
        graph.launch(stream.cuda_stream)

    for _ in range(a.warmup):
        step()
    graph.status(stream.cuda_stream)
    torch.cuda.synchronize()
    # self-check against the reference's residues for the primes it covers
    got = d_out.cpu().numpy().view(np.uint64)
    for i, r in golden_check(n, M, d, a.prime_bits).items():
        if rank == 0 and i < B:
            assert int(got[i]) == r, f"residue mismatch at prime {i}: {int(got[i])} != {r}"

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    import multi

    def max_over_ranks(x):
        return multi.max_over_ranks(x, dist, device="cuda")

    launches = 0
    barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            step()
            launches += graph.launches()
        e1.record(stream)
        barrier()
    graph.status(stream.cuda_stream)
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * B * a.steps / (ms * 1e-3)
    graph.close()  # its workspace (about 1 GiB per prime) goes back before the e2e run allocates the engine's

    # end to end through the public API with host buffers (copies inside the timed region)
    host_primes = np.array(primes, dtype=np.uint64)
    barrier()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        res = eng.residues(host_primes, n, d, queries)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * B * a.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * B + 8 * J + 4,
           "d2h_bytes_per_step": 8 * B * J + 4}
    assert np.array_equal(res.reshape(-1), got[:B * J]), "e2e residues differ from the device-timed run"

    # the plain form: one launch per prime (B = 1), the same n, M, d, one launch on the same stream
    plain = None
    if not a.no_plain_form:
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        eng.residues_async(d_primes.data_ptr(), 1, n, d, queries, d_out.data_ptr(), stream.cuda_stream)
        q1.record(stream)
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(q0.elapsed_time(q1))
        plain = {"value": world / (plain_ms * 1e-3), "unit": UNIT, "ms_per_prime": plain_ms,
                 "what": "one launch per prime (batch of 1), same n, M, d and kernel, timed alone"}

    probe = ctypes.CDLL(os.path.join(PKG, "lib", "libcuckoo_b200_probe.so"))
    probe.cfp_imad_ops_per_s.restype = ctypes.c_double
    probe.cfp_imad_ops_per_s.argtypes = [ctypes.c_int, ctypes.c_int]
    peak = probe.cfp_imad_ops_per_s(local, 5) / 1e12
    # the timed stream holds only this engine's launches, back to back: per-GPU algorithmic rate
    achieved = B * a.steps * algorithmic_mm(n) * K_OPS_PER_MM / (ms * 1e-3) / 1e12
    per_prime = MEASURED_TRAFFIC_PER_PRIME.get((n, M, d, a.prime_bits))
    traffic = a.traffic_bytes or (per_prime * B if per_prime else None)
    hbm = None
    if traffic:  # the kernel's DRAM bytes per launch (ncu) over its device-timed launch duration
        gbs = traffic / (ms / a.steps * 1e-3) / 1e9
        peak_gbs, which = hbm_peak()
        hbm = {"achieved": gbs, "peak": peak_gbs, "unit": "GB/s", "frac": gbs / peak_gbs, "peak_source": which}
    eng.close()  # its workspace (a wave of tables) goes back before the runs below allocate theirs

    def section(fn, *args, **kw):
        """A secondary measurement: its failure is reported in its own key, never in place of the
        headline line."""
        try:
            return fn(*args, **kw)
        except Exception as exc:  # noqa: BLE001 - recorded in the JSON line
            import traceback

            traceback.print_exc()
            print(f"bench: {fn.__name__} failed: {exc!r}", file=sys.stderr)
            return {"error": repr(exc)[:300]}

    solo = rank == 0 and world == 1

    def sweep_fn():
        with cb.Engine(local) as eng2:
            out = sweep_run(eng2, n, M, B)
        for v in out.values():
            v["frac"] = v["frac"] / peak if peak else None
        return out

    def cfg2_fn():
        out = config2_run(local)
        for k in ("default", "tuned"):
            out[k]["frac"] = out[k].pop("frac_top") / peak if peak else None
        return out

    def uneven_fn():
        with cb.Engine(local) as eng2:
            return uneven_run(eng2, a.uneven_stride)

    sweep = section(sweep_fn) if solo and not a.no_sweep and n == 16384 else None
    cfg2 = section(cfg2_fn) if solo and not a.no_config2 else None
    large = section(large_run, local) if solo and not a.no_large else None
    unev = section(uneven_fn) if solo and not a.no_uneven else None
    cpu = None
    if solo and not a.no_cpu_baseline and os.path.exists(reference_binary()[0]):
        cpu = section(cpu_baseline, n, M, d)
    serving = None
    if solo and not a.no_serving:
        serving = section(serving_run, local, a.serve_seconds, full_seconds=a.serve_full_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic",
            "config": {"workload": workload, "batch_primes_per_step": B, "queries_per_prime": J,
                       "l2": "inputs larger than L2 (per-prime tables total far above 126 MB)"},
            "roofline": {"bound": "int32", "achieved": achieved, "peak": peak, "unit": "Top/s (INT32 IMAD)",
                         "frac": achieved / peak if peak else None,
                         "traffic": traffic, "hbm": hbm,
                         "model": f"{K_OPS_PER_MM} INT32 multiply ops per modular multiplication, "
                                  f"{algorithmic_mm(n):.3e} multiplications per prime-residue; peak measured live"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
            "plain_form": plain, "config2": cfg2, "config3_sweep": sweep, "large_tables": large, "uneven": unev,
            "serving": serving}))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
