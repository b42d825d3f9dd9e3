#!/usr/bin/env python3
"""`cuckoo_fail single` of the reference's 32-bit library on the B200 engine.

    python cuckoo-failure_b200/single.py -n N -M M -d D [--replacement] [--exact] [--mod P] [--device K]

The reference CLI (src/cuckoo_fail.cpp:133-200) evaluates the one-table suffix DP modulo 32-bit
NTT primes on one CPU core and recombines N_bad by CRT.  Here the same primes
(cf_lib_primes: include/cuckoo/modint.hpp:183-196, src/cuckoo_fail.cpp:151-170) go to the GPU
engine in one batch (cf_residues), and crt.py recombines the residues.  The output lines follow
the reference's: the problem line, the algorithm line, "primes: k (product 2^b)  time: t s",
"p_fail = ...", "log2(p_fail) = ...,  log10(p_fail) = ...", and with --exact "N_bad = ..." and
"Q^n   = ...".  With --mod P (a prime below 2^32 with transform_length(n) | P - 1) only
"N_bad mod P = r" is printed.

The printed p_fail comes from the exact integers (the library derives it from long-double
logarithms, so the last printed digit may differ); N_bad itself is exact.
"""
import argparse
import math
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import crt  # noqa: E402
import cuckoo_b200 as cb  # noqa: E402


def solve(n, M, d, replacement=False, engine=None, device=0):
    """(primes, residues, N_bad, Q^n, seconds) for one (n, M, d) on the GPU."""
    model = cb.MODEL_REPLACEMENT if replacement else cb.MODEL_SUBSET
    primes = cb.lib_primes(n, M, d, model)
    t0 = time.perf_counter()
    own = engine is None
    eng = cb.Engine(device) if own else engine
    try:
        res = eng.residues(primes, n, d, [(n, M)], model=model).reshape(-1)
    finally:
        if own:
            eng.close()
    secs = time.perf_counter() - t0
    x, m = crt.crt(list(zip(primes, (int(r) for r in res))))
    Qn = crt.q_power(n, M, d, replacement)
    assert m > Qn and x <= Qn, (n, M, d)
    return primes, [int(r) for r in res], x, Qn, secs


def log2_exact(x):
    s = max(0, x.bit_length() - 64)
    return math.log2(x >> s) + s


def main(argv=None):
    ap = argparse.ArgumentParser(prog="single.py")
    ap.add_argument("-n", type=int, required=True)
    ap.add_argument("-M", type=int, required=True)
    ap.add_argument("-d", type=int, required=True)
    ap.add_argument("--replacement", action="store_true")
    ap.add_argument("--exact", action="store_true")
    ap.add_argument("--mod", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    n, M, d = a.n, a.M, a.d
    model = cb.MODEL_REPLACEMENT if a.replacement else cb.MODEL_SUBSET
    print(f"one table: n={n} items, M={M} slots, d={d} choices, "
          + ("d independent draws with replacement" if a.replacement else "uniform d-subset of candidate slots"))
    bits = n * crt.log2_q(M, d, a.replacement)
    print(f"algorithm: ntt (B200 engine);  outcomes Q^n = 2^{bits:.3f}")
    if a.mod:
        t0 = time.perf_counter()
        with cb.Engine(a.device) as eng:
            r = int(eng.residues([a.mod], n, d, [(n, M)], model=model)[0, 0])
        print(f"N_bad mod {a.mod} = {r}  ({time.perf_counter() - t0:.3f} s)")
        return 0
    primes, _, x, Qn, secs = solve(n, M, d, a.replacement, device=a.device)
    have = sum(math.log2(p) for p in primes)
    print(f"primes: {len(primes)} (product 2^{have:.1f})  time: {secs:.3f} s")
    if x == 0:
        print("N_bad = 0,  p_fail = 0")
        return 0
    lg = log2_exact(x) - log2_exact(Qn)
    print(f"p_fail = {x / Qn:.15e}")  # int / int is correctly rounded
    print(f"log2(p_fail) = {lg:.6f},  log10(p_fail) = {lg * math.log10(2):.6f}")
    if a.exact:
        if hasattr(sys, "set_int_max_str_digits"):
            sys.set_int_max_str_digits(0)
        print(f"N_bad = {x}")
        print(f"Q^n   = {Qn}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
