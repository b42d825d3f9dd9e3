"""The C ABI library: it loads, exports every symbol include/cuckoo_b200.h declares, and its
host helpers (prime list, need, transform length) agree with the oracle.  No GPU calls."""
import ctypes
import os
import re

import cuckoo_b200 as cb
import helpers as h

HEADER = os.path.join(h.ROOT, "include", "cuckoo_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cf_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = cb.lib()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), name


def test_prime_range_matches_oracle():
    assert cb.prime_range(0, 50) == h.oracle_primes(0, 50)
    assert cb.prime_range(1000, 7) == h.oracle_primes(1000, 7)
    assert cb.prime_range(5, 0) == []


def test_need_matches_oracle_long_double():
    o = h.oracle()
    for d in (1, 2, 3, 4):
        for n in (1, 8, 20, 200, 511, 4096, 16384):
            for M in (n + 1, 2 * n, 3 * n + 7, 4 * n):
                if d > M:
                    continue
                for model in (0, 1):
                    assert cb.need(n, M, d, model) == o.oc_need(n, M, d, model), (n, M, d, model)


def test_transform_length():
    for n in (1, 15, 16, 17, 200, 256, 257, 16384):
        assert cb.transform_length(n) == h.oracle().oc_transform_length(n)


def test_workspace_bytes_grows_quadratically():
    a, b = cb.workspace_bytes(4096, 8192, 1), cb.workspace_bytes(8192, 16384, 1)
    assert 3.5 < b / a < 4.5
    # V and S in 16 x 16 blocks at their peak live size, about n^2 / 4 words each
    n = 16384
    assert n * n // 2 * 8 <= cb.workspace_bytes(n, 2 * n, 1) < (n * n // 2 + 2 * 1024 * 1024) * 8


def test_62bit_prime_list_and_need_match_reference_output():
    """cf_prime_range_bits / cf_need_bits with 62 bits reproduce the -DFP_RB=64 reference's output:
    the same primes, and exactly need(n, M) lines per query."""
    d, queries, first, count, lines = h.load_fast_golden("fast62_small_d3.txt")
    primes = sorted({(i, p) for i, p, *_ in lines})
    assert cb.prime_range(0, count, bits=62) == [p for _, p in primes]
    assert all(p < 2**62 and p > 2**61 and (p - 1) % 2**20 == 0 for _, p in primes)
    for n, M in queries:
        got = sum(1 for ln in lines if (ln[2], ln[3]) == (n, M))
        assert got == min(count, cb.need(n, M, d, bits=62)), (n, M)
    assert cb.need(16384, 32768, 3, bits=62) < cb.need(16384, 32768, 3)  # about 20 % fewer primes
