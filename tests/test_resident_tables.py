"""Resident tables for serving (cf_tables_build / cf_tables_query).

CPU: a serving build run through the CPU harness keeps the whole V triangle (folded) and the pair
tables; unfolded, the triangle equals the oracle's suffix table entry for entry.  The query
formula of k_table_query (row sums, then the Horner finish) applied to that kept data gives the
oracle's N_bad residues for every (n' <= n, M' <= F).
GPU: queries answered from resident tables equal cf_residues' residues, for several (n', M') per
table set and both models."""
import ctypes

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

P0 = 1125899865948161


def keep_build(p, n, F, d, model):
    L = h.emu()
    words = L.emu_keep_words(n, max(n, F))
    out = np.zeros(words, dtype=np.uint64)
    rc = L.emu_keep_build(p, n, F, d, model, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    assert rc == 0
    return [int(x) for x in out]


def keep_layout(n, F):
    def take(at, cnt):
        return at, at + ((cnt + 31) & ~31)
    tri, at = take(0, n * (n + 1) // 2)
    fact, at = take(at, 2 * (F + 1))
    ifact, at = take(at, 2 * (F + 1))
    inv, at = take(at, 2 * (F + 1))
    return tri, fact, ifact, inv


def oracle_table(p, n, d, model):
    out = np.zeros(n * (n + 1) // 2, dtype=np.uint64)
    assert h.oracle().oc_suffix_table(p, n, d, model, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))) == 0
    return [int(x) for x in out]


CASES = [(40, 3, 0, 100), (70, 2, 1, 200), (300, 4, 0, 700)]


@pytest.mark.parametrize("n,d,model,F", CASES)
def test_kept_triangle_is_the_suffix_table(n, d, model, F):
    p = P0
    keep = keep_build(p, n, F, d, model)
    tri, fa, ifa, iv = keep_layout(n, F)
    fact = [keep[fa + 2 * k] for k in range(F + 1)]
    assert fact[:6] == [1, 1, 2, 6, 24, 120] and all(keep[fa + 2 * k + 1] == (fact[k] << 64) // p for k in range(F + 1))
    want = oracle_table(p, n, d, model)
    d0 = d if model == 0 else 1
    for q in range(1, n + 1):
        for w in range(d0, q):
            vs = keep[tri + q * (q - 1) // 2 + w]
            v = vs * fact[w] % p * fact[q - 1 - w] % p * fact[q - 1] % p  # unfold
            assert v == want[q * (q - 1) // 2 + w], (q, w)


@pytest.mark.parametrize("n,d,model,F", CASES)
def test_query_formula_on_kept_tables(n, d, model, F):
    """The arithmetic of k_table_query, restated on the kept words, gives the oracle's residues."""
    p = P0
    keep = keep_build(p, n, F, d, model)
    tri, fa, ifa, iv = keep_layout(n, F)
    fact = lambda k: keep[fa + 2 * k]
    ifact = lambda k: keep[ifa + 2 * k]
    inv = lambda k: keep[iv + 2 * k]
    d0 = d if model == 0 else 1
    rng = np.random.default_rng(n)
    for nq in sorted({n, max(1, n // 2), int(rng.integers(1, n + 1))}):
        Mq = int(rng.integers(nq + 1, F + 1))
        if model == 0 and d > Mq:
            continue
        ps = [0] * (nq + 1)
        for q in range(d0 + 1, nq + 1):
            ps[q] = sum(keep[tri + q * (q - 1) // 2 + w] * inv(Mq - w) for w in range(d0, q)) % p
        Q = pow(Mq, d, p) if model == 1 else fact(Mq) * ifact(d) * ifact(Mq - d) % p
        s = sum(ps[k] * inv(k) * ifact(nq - k) * ifact(Mq - k) * pow(Q, nq - k, p) for k in range(1, nq + 1)) % p
        got = s * fact(nq) % p * fact(Mq) % p
        assert got == h.oracle_residues(p, nq, d, [(nq, Mq)], model)[0], (nq, Mq)


@pytest.mark.gpu
@pytest.mark.parametrize("model", [0, 1])
def test_resident_queries_equal_direct_residues(model):
    d = 3
    for n, F, count in ((200, 800, 6), (1500, 6000, 4)):
        primes = cb.prime_range(3, count)
        rng = np.random.default_rng(n + model)
        queries = [(n, 4 * n)] + [(int(x), int(x * rng.uniform(1.5, 4)) + 1) for x in rng.integers(8, n, 5)]
        queries = [(a, min(b, F)) for a, b in queries]
        with cb.Engine(0) as eng:
            with eng.tables(primes, n, F, d, model=model) as tab:
                got = tab.query(queries)
                assert eng.last_launches() == 1
            want = eng.residues(primes, n, d, queries, model=model)
        assert np.array_equal(got, want)
