#!/usr/bin/env python3
"""Exact N_bad and p_fail from residue files by CRT, on Python integers (no gmpy2).

Drop-in for the reference's post-processing step, fast/post_gmp.py (zcy05331/Cuckoo-Failure):
same command line, same input (the engine's "i p n M residue" lines), same table on stdout.

    python cuckoo-failure_b200/crt.py D out_file... [--pbits 49] [--dump DIR] [--replacement] > table.tsv

Columns (fast/post_gmp.py:77-89):
  n, M, ratio M/n, log2_pfail (15 decimals), le_2^-40 / le_2^-64 / le_2^-128 (exact tests
  N_bad 2^lambda <= Q^n), p_fail (exact quotient N_bad / Q^n truncated to 40 significant digits),
  primes (how many residues were combined).
A query whose residues do not cover prime numbers 0 .. need-1 gets "INCOMPLETE got/need".

--pbits: every prime in the files is above 2^pbits (49 for the 50-bit engine; 31 is the
reference script's default).  --dump DIR writes N_<n>_<M>.txt with N_bad in decimal.
--replacement: Q = M^d (the library's model with d independent draws) instead of C(M, d); the
reference script has only the d-subset model.
"""
import math
import os
import sys
from collections import defaultdict
from decimal import ROUND_HALF_EVEN, Context, Decimal

HEADER = "n\tM\tratio\tlog2_pfail\tle_2^-40\tle_2^-64\tle_2^-128\tp_fail\tprimes"


def read_residues(paths):
    """{(n, M): {prime number i: (p, residue)}} from output files (fast/post_gmp.py:36-42)."""
    res = defaultdict(dict)
    for fn in paths:
        with open(fn) as f:
            for line in f:
                t = line.split()
                if len(t) == 5:
                    res[(int(t[2]), int(t[3]))][int(t[0])] = (int(t[1]), int(t[4]))
    return res


def log2_q(M, d, replacement=False):
    """log2 Q in double precision: sum of log2(M-i) - log2(i+1) (fast/post_gmp.py:46), or d log2 M."""
    if replacement:
        return d * math.log2(M)
    return sum(math.log2(M - i) - math.log2(i + 1) for i in range(d))


def need(n, M, d, pbits, replacement=False):
    """Residues a query needs: ceil((n log2 Q + 3) / pbits) + 1 (fast/post_gmp.py:45-47)."""
    return math.ceil((n * log2_q(M, d, replacement) + 3) / float(pbits)) + 1


def crt(pairs):
    """(x, m) with x = r_k mod p_k for every (p_k, r_k), 0 <= x < m = prod p_k.

    Pairwise merging up a balanced tree (fast/post_gmp.py:50-60): merging (x1, m1) with (x2, m2)
    gives x1 + m1 ((x2 - x1) m1^-1 mod m2), which stays canonical, so the result does not depend
    on the merge order."""
    items = [(r % p, p) for p, r in pairs]
    if not items:
        return 0, 1
    while len(items) > 1:
        nxt = []
        for k in range(0, len(items) - 1, 2):
            (x1, m1), (x2, m2) = items[k], items[k + 1]
            nxt.append((x1 + m1 * ((x2 - x1) * pow(m1, -1, m2) % m2), m1 * m2))
        if len(items) % 2:
            nxt.append(items[-1])
        items = nxt
    return items[0]


class PrefixCRT:
    """CRT over prefixes of one fixed prime list, with the big-integer constants cached.

    Every query's primes are primes number 0 .. k-1 of the same list, so the merge tree can be
    fixed once: [0, k) splits into dyadic blocks [s, s + 2^l) (the binary digits of k, largest
    first), each block merges its halves recursively, and the blocks merge left to right.  The
    block products and the modular inverses of each merge (m_left^-1 mod m_right) depend only on
    the list, so they are computed once and reused; a query then costs multiplications and
    reductions only, no extended Euclid.  The result equals crt() (both are the canonical residue)."""

    def __init__(self, primes):
        self.p = [int(q) for q in primes]
        self._prod = {}
        self._inv = {}

    def prod(self, lo, hi):
        key = (lo, hi)
        m = self._prod.get(key)
        if m is None:
            if hi - lo == 1:
                m = self.p[lo]
            else:
                mid = (lo + hi) // 2
                m = self.prod(lo, mid) * self.prod(mid, hi)
            self._prod[key] = m
        return m

    def _merge_inv(self, key, ml, mr):
        v = self._inv.get(key)
        if v is None:
            v = pow(ml % mr, -1, mr)
            self._inv[key] = v
        return v

    def _block(self, lo, hi, r):
        if hi - lo == 1:
            return r[lo] % self.p[lo]
        mid = (lo + hi) // 2
        xl, xr = self._block(lo, mid, r), self._block(mid, hi, r)
        ml, mr = self.prod(lo, mid), self.prod(mid, hi)
        return xl + ml * ((xr - xl) * self._merge_inv(("b", lo, hi), ml, mr) % mr)

    def crt(self, residues):
        """(x, m) for residues r_0 .. r_{k-1} modulo primes 0 .. k-1 of the list."""
        r = [int(v) for v in residues]
        k = len(r)
        if k > len(self.p):
            raise ValueError("more residues than primes")
        x, m, s = 0, 1, 0
        for lvl in range(k.bit_length() - 1, -1, -1):
            if not (k >> lvl) & 1:
                continue
            e = s + (1 << lvl)
            xb, mb = self._block(s, e, r), self.prod(s, e)
            if s == 0:
                x, m = xb, mb
            else:
                x = x + m * ((xb - x) * self._merge_inv(("p", s, e), m, mb) % mb)
                m = m * mb
            s = e
        return x, m


def q_power(n, M, d, replacement=False):
    """Q^n exactly: C(M, d)^n, or (M^d)^n for the replacement model."""
    return (M**d if replacement else math.comb(M, d)) ** n


def _log2_big(x, ctx):
    """log2 of a positive integer to about 60 significant digits (the top 200 bits suffice)."""
    s = max(0, x.bit_length() - 200)
    top = x >> s
    return ctx.divide(ctx.ln(Decimal(top)), ctx.ln(Decimal(2))) + s


def log2_ratio_text(x, D):
    """log2(x / D) rounded to 15 decimals, as text ("-inf" for x = 0)."""
    if x == 0:
        return "-inf"
    ctx = Context(prec=60)
    v = ctx.subtract(_log2_big(x, ctx), _log2_big(D, ctx))
    return format(v.quantize(Decimal("1e-15"), rounding=ROUND_HALF_EVEN, context=ctx), "f")


def sci(N, D, digits=40):
    """N / D truncated to `digits` significant digits as "d.ddd...e<exp>" (fast/post_gmp.py:63-74),
    by exact integer arithmetic."""
    if N == 0:
        return "0"
    # exponent e = floor(log10(N / D)): estimate from the bit lengths, then correct exactly
    e = math.floor((N.bit_length() - D.bit_length()) * math.log10(2))

    def below(k):  # N / D < 10^k
        return N * 10 ** (-k) < D if k <= 0 else N < D * 10**k

    while not below(e + 1):
        e += 1
    while below(e):
        e -= 1
    s = digits - 1 - e
    q = N * 10**s // D if s >= 0 else N // (D * 10 ** (-s))
    t = str(q)
    assert len(t) == digits
    return t[0] + "." + t[1:] + "e%d" % e


def table_rows(res, d, pbits, replacement=False, dump=None):
    """The output lines, one per (n, M) in sorted order (fast/post_gmp.py:77-93)."""
    yield HEADER
    for n, M in sorted(res):
        got = res[(n, M)]
        k = need(n, M, d, pbits, replacement)
        if any(i not in got for i in range(k)):
            yield f"{n}\t{M}\t{M / n:.6f}\tINCOMPLETE {len(got)}/{k}"
            continue
        x, m = crt([got[i] for i in range(k)])
        Qn = q_power(n, M, d, replacement)
        # the primes' product must exceed Q^n >= N_bad with room to spare, and N_bad <= Q^n
        assert m > 4 * Qn and x <= Qn, (n, M)
        tests = "\t".join("yes" if (x << lam) <= Qn else "no" for lam in (40, 64, 128))
        yield f"{n}\t{M}\t{M / n:.6f}\t{log2_ratio_text(x, Qn)}\t{tests}\t{sci(x, Qn)}\t{k}"
        if dump:
            write_dump(dump, n, M, d, x, replacement)


def write_dump(directory, n, M, d, x, replacement=False):
    limit = sys.get_int_max_str_digits() if hasattr(sys, "get_int_max_str_digits") else None
    if limit is not None:
        sys.set_int_max_str_digits(0)
    try:
        q = f"({M}^{d})^{n}" if replacement else f"C({M},{d})^{n}"
        with open(os.path.join(directory, f"N_{n}_{M}.txt"), "w") as f:
            f.write("N_bad=" + str(x) + f"\nQ^n={q}\n")
    finally:
        if limit is not None:
            sys.set_int_max_str_digits(limit)


def main(argv=None):
    args = list(sys.argv[1:] if argv is None else argv)
    dump, pbits, replacement = None, 31, False
    if "--pbits" in args:
        k = args.index("--pbits")
        pbits = int(args[k + 1])
        del args[k:k + 2]
    if "--dump" in args:
        k = args.index("--dump")
        dump = args[k + 1]
        del args[k:k + 2]
    if "--replacement" in args:
        args.remove("--replacement")
        replacement = True
    if not args:
        print(__doc__.strip().splitlines()[3].strip(), file=sys.stderr)
        return 2
    d = int(args[0])
    for line in table_rows(read_residues(args[1:]), d, pbits, replacement, dump):
        print(line)
        sys.stdout.flush()
    return 0


if __name__ == "__main__":
    sys.exit(main())
