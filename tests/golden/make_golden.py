#!/usr/bin/env python3
"""Regenerate the golden fixtures in this directory from the reference's own programs.

The fixtures are outputs of the reference (zcy05331/Cuckoo-Failure) built from its sources by
oracle/Makefile.ref into oracle/_ref/: the 64-bit batch engine's host build
(fast/cuckoo_fast.cu, byte-identical scalar and AVX-512 IFMA builds, and the scalar build with
62-bit primes, -DFP_RB=64) and the 32-bit library CLI (src/cuckoo_fail.cpp).  They pin the oracle and the CUDA engine to the reference.

Run from the repository root, where the reference tree is available:
    make -f oracle/Makefile.ref && python tests/golden/make_golden.py
"""
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


def run_fast(d, queries, first, count, out_name, batch=None, binary=None):
    """fast/cuckoo_fast.cu CLI: cuckoo_fast D QUERIES FIRST COUNT [--batch B] -> 'i p n M residue' lines."""
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        for n, M in queries:
            f.write(f"{n} {M}\n")
        qpath = f.name
    cmd = [binary or fast_bin(), str(d), qpath, str(first), str(count)]
    if batch:
        cmd += ["--batch", str(batch)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    os.unlink(qpath)
    with open(os.path.join(HERE, out_name), "w") as g:
        g.write(f"# d={d} queries={' '.join(f'{n},{M}' for n, M in queries)} first={first} count={count}\n")
        g.write(out)
    print(out_name, len(out.splitlines()), "lines")


def run_lib(args):
    return subprocess.run([os.path.join(REF, "cuckoo_fail")] + args, check=True, capture_output=True, text=True).stdout


def main():
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
