#!/usr/bin/env python3
"""Regenerate the golden fixtures in this directory from the reference's own programs.

The fixtures are outputs of the reference (zcy05331/Cuckoo-Failure) built from its sources by
oracle/Makefile.ref into oracle/_ref/: the 64-bit batch engine's host build
(fast/cuckoo_fast.cu, byte-identical scalar and AVX-512 IFMA builds, and the scalar build with
62-bit primes, -DFP_RB=64) and the 32-bit library CLI (src/cuckoo_fail.cpp).  They pin the oracle and the CUDA engine to the reference.

Run from the repository root, where the reference tree is available:
    make -f oracle/Makefile.ref && python tests/golden/make_golden.py [--groups base,large]

Groups: `base` (small sizes, config 2, one or two primes at n = 16384, the library CLI at small n),
`large` (the replacement model at n = 4096 and 16384 through the library's --mod P, 18 queries
at n <= 16384, and a seeded sample of the uneven-batch workload) and `huge` (tables above
n = 16384: n = 32768 and n = 65536, primes 0 and 1, one host-build process per prime, and
n = 32768 with 62-bit primes; the n = 65536 runs take 32 GB of host memory each and run one after
the other).
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")


def fast_bin():
    ifma = os.path.join(REF, "cuckoo_fast_ifma")
    has_ifma = "avx512ifma" in open("/proc/cpuinfo").read()
    return ifma if has_ifma and os.path.exists(ifma) else os.path.join(REF, "cuckoo_fast_cpu")


def fast_lines(d, queries, first, count, batch=None, binary=None):
    """fast/cuckoo_fast.cu CLI: cuckoo_fast D QUERIES FIRST COUNT [--batch B] -> its stdout
    ('i p n M residue' lines)."""
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        for n, M in queries:
            f.write(f"{n} {M}\n")
        qpath = f.name
    cmd = [binary or fast_bin(), str(d), qpath, str(first), str(count)]
    if batch:
        cmd += ["--batch", str(batch)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    os.unlink(qpath)
    return out


def run_fast(d, queries, first, count, out_name, batch=None, binary=None):
    out = fast_lines(d, queries, first, count, batch, binary)
    with open(os.path.join(HERE, out_name), "w") as g:
        g.write(f"# d={d} queries={' '.join(f'{n},{M}' for n, M in queries)} first={first} count={count}\n")
        g.write(out)
    print(out_name, len(out.splitlines()), "lines")


def run_lib(args):
    return subprocess.run([os.path.join(REF, "cuckoo_fail")] + args, check=True, capture_output=True, text=True).stdout


def lib_mod(n, M, d, P, rep):
    """`cuckoo_fail single ... --mod P` -> the residue line of lib_cuckoo_fail.txt's 'mod' form."""
    t = run_lib(["single", "-n", str(n), "-M", str(M), "-d", str(d), "--mod", str(P)] + (["--replacement"] if rep else []))
    r = re.search(r"N_bad mod (\d+) = (\d+)", t)
    return f"mod {int(rep)} {n} {M} {d} {r.group(1)} {r.group(2)}"


def large():
    """Full-size pins: the replacement model (no 50-bit reference exists, the fast engine hard-codes
    C(v, d)) through the library at the primes it would choose itself; 18 queries at n <= 16384
    against the host build; a seeded sample of the uneven-batch workload."""
    sys.path.insert(0, os.path.join(ROOT, "cuckoo-failure_b200"))
    import numpy as np

    import cuckoo_b200 as cb
    import uneven

    jobs = {}
    with cf.ThreadPoolExecutor(max(1, (os.cpu_count() or 2) - 1)) as ex:
        # 1. library --mod P: the first two primes of the library's own list for each case
        for n, M, d, rep in ((16384, 32768, 3, True), (4096, 8192, 3, True), (4096, 8192, 3, False)):
            for P in cb.lib_primes(n, M, d, int(rep))[:2]:
                jobs[("lib", n, M, d, P, rep)] = ex.submit(lib_mod, n, M, d, P, rep)
        # 2. 18 queries with n in [1000, 16384] (16384 included), M in [1.5 n, 4 n], primes 0 and 1
        rng = np.random.default_rng(18)
        ns = [16384] + sorted({int(x) for x in np.exp(rng.uniform(np.log(1000), np.log(16384), 17))}, reverse=True)
        qJ = [(n, int(round(n * rng.uniform(1.5, 4.0)))) for n in ns]
        jobs[("J18",)] = ex.submit(fast_lines, 3, qJ, 0, 2)
        # 3. the first 16 instances of the uneven-batch workload, grouped by d as one table set per d
        #    serves them: primes 0 and 1 (every instance active), and each instance's last prime
        #    need - 1 (only the instances that still need it active)
        insts = uneven.instances(16)
        byd = {}
        for n, M, d in insts:
            byd.setdefault(d, []).append((n, M))
        for d, qs in byd.items():
            jobs[("unev", d, 0)] = ex.submit(fast_lines, d, qs, 0, 2)
            for n, M in qs:
                k = cb.need(n, M, d) - 1
                if ("unev", d, k) not in jobs:
                    jobs[("unev", d, k)] = ex.submit(fast_lines, d, qs, k, 1)
        res = {k: f.result() for k, f in jobs.items()}
    with open(os.path.join(HERE, "lib_large.txt"), "w") as g:
        g.write("# 'mod rep n M d P residue' from the library CLI (cuckoo_fail single ... --mod P), P among the "
                "first primes of the library's own list for (n, M, d)\n")
        g.write("".join(v + "\n" for k, v in sorted(res.items(), key=lambda kv: str(kv[0])) if k[0] == "lib"))
    with open(os.path.join(HERE, "fast_n16384_d3_J18.txt"), "w") as g:
        g.write(f"# d=3 queries={' '.join(f'{n},{M}' for n, M in qJ)} first=0 count=2\n")
        g.write(res[("J18",)])
    with open(os.path.join(HERE, "uneven_sample.txt"), "w") as g:
        g.write(f"# uneven.instances(16) (seed {uneven.CONFIG4_SEED}): "
                + " ".join(f"{n},{M},{d}" for n, M, d in insts) + "\n")
        g.write("# 'd i p n M residue' from the host build, one run per d over that d's instances\n")
        for k in sorted(k for k in res if k[0] == "unev"):
            for ln in res[k].splitlines():
                g.write(f"{k[1]} {ln}\n")
    print("large fixtures written")


def huge():
    """Tables above n = 16384 (transform lengths 2^15 and 2^16), d = 3, primes 0 and 1; and the
    headline size n = 16384 for primes 0 .. 15 (one process per prime)."""
    with cf.ThreadPoolExecutor(max(1, (os.cpu_count() or 2))) as ex:
        outs = list(ex.map(lambda i: fast_lines(3, [(16384, 32768)], i, 1), range(16)))
    with open(os.path.join(HERE, "fast_n16384_d3_first16.txt"), "w") as g:
        g.write("# d=3 queries=16384,32768 first=0 count=16 (one run per prime)\n")
        g.write("".join(outs))
    for n, queries, parallel in ((32768, [(32768, 65536), (20000, 50000)], True), (65536, [(65536, 131072)], False)):
        if parallel:
            with cf.ThreadPoolExecutor(2) as ex:
                outs = list(ex.map(lambda i: fast_lines(3, queries, i, 1), (0, 1)))
        else:
            outs = [fast_lines(3, queries, i, 1) for i in (0, 1)]
        name = f"fast_n{n}_d3.txt"
        with open(os.path.join(HERE, name), "w") as g:
            g.write(f"# d=3 queries={' '.join(f'{a},{b}' for a, b in queries)} first=0 count=2 (one run per prime)\n")
            g.write("".join(outs))
        print(name, sum(len(o.splitlines()) for o in outs), "lines")
    # the reference's published case at n = 65536 has 126 queries (fast/README.md:80-86): a seeded
    # set of 126 (n, M), n log-uniform in [2000, 65536] with 65536 itself, M = n U[1.5, 4]; prime 0
    import numpy as np

    rng = np.random.default_rng(126)
    ns = [65536] + sorted({int(x) for x in np.exp(rng.uniform(np.log(2000), np.log(65536), 140))}, reverse=True)
    q126 = [(n, int(round(n * rng.uniform(1.5, 4.0)))) for n in ns[:126]]
    with open(os.path.join(HERE, "fast_n65536_d3_J126.txt"), "w") as g:
        g.write(f"# d=3 queries={' '.join(f'{a},{b}' for a, b in q126)} first=0 count=1\n")
        g.write(fast_lines(3, q126, 0, 1))
    # 62-bit primes (-DFP_RB=64) at n = 32768, primes 0 and 1
    b64 = os.path.join(REF, "cuckoo_fast_cpu64")
    q = [(32768, 65536), (20000, 50000)]
    with cf.ThreadPoolExecutor(2) as ex:
        outs = list(ex.map(lambda i: fast_lines(3, q, i, 1, binary=b64), (0, 1)))
    with open(os.path.join(HERE, "fast62_n32768_d3.txt"), "w") as g:
        g.write(f"# d=3 queries={' '.join(f'{a},{b}' for a, b in q)} first=0 count=2 (one run per prime)\n")
        g.write("".join(outs))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--groups", default="base,large")
    groups = ap.parse_args().groups.split(",")
    if "huge" in groups:
        huge()
    if "large" in groups:
        large()
    if "base" not in groups:
        return 0
    small = [(8, 9), (8, 20), (37, 50), (100, 150), (200, 400), (255, 256), (256, 600), (300, 301), (512, 1024)]
    for d in (2, 3, 4):
        run_fast(d, small, 0, 40, f"fast_small_d{d}.txt")
    # non-power-of-two nmax, different first prime, tiny n
    run_fast(3, [(9, 10), (13, 40), (300, 700)], 17, 6, "fast_n300_first17.txt")
    run_fast(1, [(8, 20), (12, 20), (50, 60)], 0, 8, "fast_d1.txt")
    # batch scale: config of the batch-scale plain method (n=4096, M=8192, d=3)
    run_fast(3, [(4096, 8192)], 0, 4, "fast_n4096_d3.txt")
    # the headline size (n=16384, M=2n) for d = 2, 3, 4, prime 0 (and prime 1 for d = 3)
    for d, cnt in ((2, 1), (3, 2), (4, 1)):
        run_fast(d, [(16384, 32768)], 0, cnt, f"fast_n16384_d{d}.txt")

    # 62-bit primes (-DFP_RB=64): small sizes, config 2, and the headline size for prime 0
    b64 = os.path.join(REF, "cuckoo_fast_cpu64")
    run_fast(3, small, 0, 24, "fast62_small_d3.txt", binary=b64)
    run_fast(2, [(4096, 8192), (1000, 3000)], 0, 2, "fast62_n4096_d2.txt", binary=b64)
    run_fast(3, [(16384, 32768)], 0, 1, "fast62_n16384_d3.txt", binary=b64)

    # 32-bit library CLI: N_bad mod P and exact N_bad (config 1 and the replacement model)
    lines = []
    for rep in (False, True):
        for n, M, d in ((20, 40, 3), (200, 400, 3), (60, 100, 2), (24, 60, 4), (6, 7, 2)):
            extra = ["--replacement"] if rep else []
            txt = run_lib(["single", "-n", str(n), "-M", str(M), "-d", str(d), "--exact"] + extra)
            nb = re.search(r"N_bad = (\d+)", txt)
            pf = re.search(r"p_fail = (\S+)", txt)
            npr = re.search(r"primes: (\d+)", txt)
            nbad = nb.group(1) if nb else "0"
            lines.append(f"exact {int(rep)} {n} {M} {d} {npr.group(1) if npr else 0} {pf.group(1) if pf else '0'} {nbad}")
            for P in (998244353, 1004535809, 4194304001):
                t = run_lib(["single", "-n", str(n), "-M", str(M), "-d", str(d), "--mod", str(P)] + extra)
                r = re.search(r"N_bad mod (\d+) = (\d+)", t)
                lines.append(f"mod {int(rep)} {n} {M} {d} {r.group(1)} {r.group(2)}")
    with open(os.path.join(HERE, "lib_cuckoo_fail.txt"), "w") as g:
        g.write("# kind replacement n M d ... : 'exact rep n M d primes p_fail N_bad' | 'mod rep n M d P residue'\n")
        g.write("\n".join(lines) + "\n")
    print("lib_cuckoo_fail.txt", len(lines), "lines")


if __name__ == "__main__":
    sys.exit(main())
