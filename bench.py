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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuckoo-failure_b200")
sys.path.insert(0, PKG)

METRIC = "prime-residues/s, n=16384 d=3 NTT suffix build; served-query p50/p99 latency"
UNIT = "prime-residues/s"
K_OPS_PER_MM = 20  # INT32 multiply ops per 64-bit modular multiplication (fixed accounting model)
# DRAM bytes (read + write) per launch of the engine kernel, from the ncu launch list of this
# bench's own command (profiles/k_suffix_n16384_b148_launches.md), keyed by (n, M, d, primes per
# launch, prime bits)
MEASURED_TRAFFIC = {(16384, 32768, 3, 148, 50): 1299.2e9 + 865.1e9}
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
    """Known residues of the reference host build for primes 0 and 1 (tests/golden)."""
    path = os.path.join(ROOT, "tests", "golden", f"fast{'62' if bits == 62 else ''}_n{n}_d{d}.txt")
    if not os.path.exists(path):
        return {}
    out = {}
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if len(t) == 5 and not ln.startswith("#") and int(t[2]) == n and int(t[3]) == M:
                out[int(t[0])] = int(t[4])
    return out


def serving_run(device, seconds, rate=200.0, n_lo=64, n_hi=2048, budget_gb=150.0, plain_sample=16):
    """Served-query latency: a seeded Poisson stream (rate per second, n log-uniform in [n_lo, n_hi],
    M = n U[1.5, 4], d in {2, 3, 4}) through serve.py's continuous-batching loop over resident
    tables built before the clock starts for (n_hi, 4 n_hi, d).  Latencies from arrival to residues
    ready (GPU) and to exact N_bad (after the host CRT pool).  Beside it the plain form on a sample
    of the same requests: each rebuilt alone (cf_residues over its primes), to residues ready."""
    import numpy as np

    import cuckoo_b200 as cb
    import serve

    stream = serve.poisson_stream(seconds, rate, n_lo, n_hi, seed=20261203)
    warm = [(n_hi, 4 * n_hi, dd) for dd in (2, 3, 4)]
    with cb.Engine(device) as eng:
        t0 = time.perf_counter()
        kmax = max(cb.need(n, M, dd) for _, n, M, dd in stream)
        pool = serve.crt_pool(kmax)
        srv_lat, _, stats = serve.run(stream, eng, budget_gb * 1e9, warm=warm, pool=pool)
        pool.shutdown()
        total = time.perf_counter() - t0
        plain = []
        for _, n, M, dd in stream[:: max(1, len(stream) // plain_sample)][:plain_sample]:
            s0 = time.perf_counter()
            eng.residues(cb.prime_range(0, cb.need(n, M, dd)), n, dd, [(n, M)])
            plain.append(time.perf_counter() - s0)
    nb = serve.percentiles(srv_lat)
    rl = stats["residues_latency"]
    warm_builds = sum((cb.need(*w, cb.MODEL_SUBSET) + serve.CHUNK - 1) // serve.CHUNK for w in warm)
    return {"workload": f"Poisson {rate:g} req/s for {seconds:g} s, n log-uniform [{n_lo}, {n_hi}], M/n U[1.5, 4], "
                        f"d in {{2,3,4}}; tables resident (built before the clock) under a {budget_gb:g} GB budget",
            "p50_ms": rl.get("p50_ms"), "p99_ms": rl.get("p99_ms"), "latency_to": "residues ready",
            "nbad_p50_ms": nb.get("p50_ms"), "nbad_p99_ms": nb.get("p99_ms"),
            "requests": stats["requests"], "rounds": stats["rounds"], "requests_per_s": stats["requests"] / stats["wall_s"],
            "builds_during_stream": stats["builds"] - warm_builds, "plain_path_requests": stats["plain"],
            "resident_gb": stats["resident_gb"], "engine_s": stats["engine_s"], "warmup_and_stream_s": total,
            "plain_rebuild_p50_ms": 1e3 * float(np.median(plain)) if plain else None, "plain_sample": len(plain),
            "note": "n above ~2048 cannot stay resident for d = 2..4 within the budget (a table at n = 16384 is "
                    "1.07 GB per prime, 14184 primes at d = 3); such requests take the plain path"}


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
    indices that are multiples of `stride` (a sample whose tables follow the whole run's mix).
    Timed as one graph of work-queue launches, beside the plain form: each instance alone, one
    cf_residues call (a launch per chunk of primes) per instance, on the first per_instance_count
    instances and the same prime indices."""
    import numpy as np
    import torch

    import cuckoo_b200 as cb
    import uneven

    insts = uneven.instances(512, seed=seed or uneven.CONFIG4_SEED)
    needs = [cb.need(n, M, d) for n, M, d in insts]
    planned = [len(range(0, k, stride)) for k in needs]
    stream = torch.cuda.Stream()
    with eng.uneven(insts, stride=stride) as u:
        ms = timed_replays(u.launch, stream, 1)
        res = u.results(stream.cuda_stream)
        tables, launches = u.tables(), u.launches()
    full_tables = len(cb.uneven_describe(insts))
    sub = insts[:per_instance_count]
    t0 = time.perf_counter()
    alone = uneven.per_instance(eng, sub, cb.prime_range, cb.need, stride=stride)
    plain_s = time.perf_counter() - t0
    for k in range(len(sub)):  # the same residues both ways
        assert [int(x) for x in res[k][::stride]] == alone[k][::stride], f"uneven instance {k} differs"
    sub_residues = sum(planned[:per_instance_count])
    sub_share = sub_residues / max(1, sum(planned))
    return {"workload": "512 instances, n log-uniform [256, 16384], M = n U{2,3,4}, d U{2,3,4}, "
                        f"seed {uneven.CONFIG4_SEED}; prime indices i = 0 mod {stride} of each instance's need",
            "tables": tables, "tables_full_run": full_tables, "launches_per_graph": launches,
            "instance_residues": sum(planned), "ms": ms,
            "instance_residues_per_s": sum(planned) / (ms * 1e-3), "tables_per_s": tables / (ms * 1e-3),
            "full_run_s_est": full_tables / (tables / (ms * 1e-3)),
            "per_instance_form": {"instances": per_instance_count, "instance_residues": sub_residues,
                                  "s": plain_s, "instance_residues_per_s": sub_residues / plain_s,
                                  "full_run_s_est": plain_s / sub_share,
                                  "what": "each instance alone: one cf_residues call over its planned primes, its own n"}}


def sweep_run(eng, n, M, B, reps=2):
    """Config-3 sweep at n = 16384, M = 2n: d = 2 and 4 (subset model) and the replacement model at
    d = 3, one graph-captured 148-prime launch per step, the residues of primes 0 and 1 checked
    where the reference has them."""
    import numpy as np
    import torch

    import cuckoo_b200 as cb

    out = {}
    stream = torch.cuda.Stream()
    for d, model in ((2, cb.MODEL_SUBSET), (4, cb.MODEL_SUBSET), (3, cb.MODEL_REPLACEMENT)):
        primes = cb.prime_range(0, B)
        d_primes = torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64), device="cuda")
        d_out = torch.empty(B, dtype=torch.int64, device="cuda")
        g = eng.batch_graph(d_primes.data_ptr(), B, n, d, [(n, M)], d_out.data_ptr(), model=model)
        ms = timed_replays(g.launch, stream, reps)
        g.status(stream.cuda_stream)
        g.close()
        got = d_out.cpu().numpy().view(np.uint64)
        if model == cb.MODEL_SUBSET:
            for i, r in golden_check(n, M, d).items():
                assert int(got[i]) == r, f"d={d}: residue mismatch at prime {i}"
        key = f"d{d}" + ("_replacement" if model else "")
        out[key] = {"value": B / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": reps,
                    "primes_needed": cb.need(n, M, d, model),
                    "frac": B * algorithmic_mm(n) * K_OPS_PER_MM / (ms * 1e-3) / 1e12}
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
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch (512 instances) run")
    ap.add_argument("--uneven-stride", type=int, default=97)
    ap.add_argument("--no-sweep", action="store_true", help="skip d = 2, 4 and the replacement model")
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
    traffic = a.traffic_bytes or MEASURED_TRAFFIC.get((n, M, d, B, a.prime_bits))
    hbm = None
    if traffic:  # the kernel's DRAM bytes per launch (ncu) over its device-timed launch duration
        gbs = traffic / (ms / a.steps * 1e-3) / 1e9
        peak_gbs, which = hbm_peak()
        hbm = {"achieved": gbs, "peak": peak_gbs, "unit": "GB/s", "frac": gbs / peak_gbs, "peak_source": which}
    eng.close()  # its workspace (a wave of tables) goes back before the runs below allocate theirs
    sweep = None
    if rank == 0 and world == 1 and not a.no_sweep and n == 16384:
        with cb.Engine(local) as eng2:
            sweep = sweep_run(eng2, n, M, B)
        for v in sweep.values():
            v["frac"] = v["frac"] / peak if peak else None
    unev = None
    if rank == 0 and world == 1 and not a.no_uneven:
        with cb.Engine(local) as eng2:
            unev = uneven_run(eng2, a.uneven_stride)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline and os.path.exists(reference_binary()[0]):
        cpu = cpu_baseline(n, M, d)
    serving = None
    if rank == 0 and world == 1 and not a.no_serving:
        serving = serving_run(local, a.serve_seconds)
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
            "plain_form": plain, "config3_sweep": sweep, "uneven": unev, "serving": serving}))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
