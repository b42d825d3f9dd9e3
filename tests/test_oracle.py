"""The oracle (a C restatement of the reference algorithm) pinned against the reference's own
outputs: golden residues from fast/cuckoo_fast.cu's host build and from the 32-bit library CLI."""
import math

import pytest

import helpers as h


def by_prime(name):
    d, queries, first, count, lines = h.load_fast_golden(name)
    exp = h.expected_by_prime(lines)
    return d, queries, exp


@pytest.mark.parametrize("name", ["fast_small_d2.txt", "fast_small_d3.txt", "fast_small_d4.txt",
                                  "fast_n300_first17.txt", "fast_d1.txt", "fast62_small_d3.txt"])
def test_oracle_matches_reference_fast_engine(name):
    d, queries, exp = by_prime(name)
    nmax = max(n for n, _ in queries)
    checked = 0
    for (i, p), want in sorted(exp.items())[:12]:
        qs = sorted(want)
        got = h.oracle_residues(p, nmax, d, qs)
        assert dict(zip(qs, got)) == want, (name, i)
        checked += len(qs)
    assert checked > 0


def test_oracle_n4096_prime1():
    d, queries, exp = by_prime("fast_n4096_d3.txt")
    (i, p), want = sorted(exp.items())[1]
    assert h.oracle_residues(p, 4096, d, [(4096, 8192)]) == [want[(4096, 8192)]]


def test_oracle_prime_list_and_need():
    # first primes of the fixed list (from the golden files) and need() values of the configs
    _, _, exp = by_prime("fast_small_d3.txt")
    primes = [p for (i, p) in sorted(exp)]
    assert h.oracle_primes(0, len(primes)) == primes
    assert h.oracle_primes(17, 3) == [p for (i, p) in sorted(by_prime("fast_n300_first17.txt")[2])][:3]
    o = h.oracle()
    assert o.oc_need(200, 400, 3, 0) == 97
    assert o.oc_need(4096, 8192, 3, 0) == 3046
    assert [o.oc_need(16384, 32768, d, 0) for d in (2, 3, 4)] == [9698, 14184, 18530]
    assert [o.oc_transform_length(n) for n in (1, 8, 16, 17, 200, 256, 4096, 16384)] == [16, 16, 16, 32, 256, 256, 4096, 16384]


def test_oracle_matches_library_cli_mod_residues():
    """N_bad mod P from the 32-bit library CLI (src/cuckoo_fail.cpp --mod), both models."""
    for rec in h.load_lib_golden():
        if rec[0] != "mod":
            continue
        _, rep, n, M, d, P, r = rec
        assert h.oracle_residues(P, n, d, [(n, M)], model=rep) == [r], rec


def test_library_exact_values_are_consistent_with_mod_residues():
    recs = h.load_lib_golden()
    exact = {(r[1], r[2], r[3], r[4]): r[7] for r in recs if r[0] == "exact"}
    for rec in recs:
        if rec[0] == "mod":
            _, rep, n, M, d, P, r = rec
            assert exact[(rep, n, M, d)] % P == r


def test_oracle_cubic_equals_ntt():
    p = h.oracle_primes(0, 1)[0]
    for model in (0, 1):
        for nmax, d, qs in ((30, 2, [(30, 40), (12, 13)]), (33, 3, [(33, 90)]), (24, 4, [(24, 60)])):
            assert h.oracle_residues(p, nmax, d, qs, model, cubic=True) == h.oracle_residues(p, nmax, d, qs, model)


def test_oracle_birthday_closed_form():
    """d = 1: N_bad = M^n - M!/(M-n)! (src/check.cpp:122-146), both sampling models."""
    p = h.oracle_primes(0, 1)[0]
    for n in (3, 7, 12):
        M = 20
        want = int(h.oracle().oc_birthday(p, n, M))
        assert want == (pow(M, n, p) - math.perm(M, n)) % p
        for model in (0, 1):
            assert h.oracle_residues(p, n, 1, [(n, M)], model) == [want]


def test_oracle_exact_crt_small():
    """CRT over the library's primes reproduces N_bad exactly (n=20, M=40, d=3: README example)."""
    rec = [r for r in h.load_lib_golden() if r[0] == "exact" and r[1:5] == (0, 20, 40, 3)][0]
    nbad = rec[7]
    ps = h.oracle_primes(0, 6)
    x, m = 0, 1
    for p in ps:
        r = h.oracle_residues(p, 20, 3, [(20, 40)])[0]
        assert r == nbad % p
        t = ((r - x) * pow(m, -1, p)) % p
        x, m = x + m * t, m * p
    assert x == nbad


def test_oracle_62bit_n4096():
    """The reference built with -DFP_RB=64 (primes below 2^62, Montgomery R = 2^64)."""
    d, queries, exp = by_prime("fast62_n4096_d2.txt")
    for (i, p), want in sorted(exp.items()):
        qs = sorted(want)
        assert dict(zip(qs, h.oracle_residues(p, 4096, d, qs))) == want
