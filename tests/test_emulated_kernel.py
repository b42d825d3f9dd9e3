"""The engine's per-prime phase code (the same source the CUDA kernel compiles) executed on the
CPU thread by thread, against the oracle and the reference's golden residues.  This checks the
transform passes, the stage index arithmetic and the query/Horner phases without a GPU."""
import pytest

import helpers as h

P0 = 1125899865948161


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("nmax,d,queries", [
    (1, 2, [(1, 2)]), (5, 1, [(5, 9)]), (8, 2, [(8, 9), (5, 20)]), (16, 3, [(16, 17), (10, 30)]),
    (20, 3, [(20, 40)]), (33, 3, [(33, 99)]), (64, 1, [(64, 100)]), (200, 3, [(200, 400), (64, 200)]),
    (256, 4, [(256, 600), (100, 101)]), (300, 2, [(300, 301), (3, 4)]),
])
def test_emulated_kernel_matches_oracle(nmax, d, queries, model):
    assert h.emu_residues([P0], nmax, d, queries, model)[0] == h.oracle_residues(P0, nmax, d, queries, model)


def test_emulated_kernel_large_geometries():
    """L = 1024 (32 entries per thread, five-level register passes, as at 2^14) and L = 2048
    (16 entries per thread, four-level passes, as at 2^11 .. 2^13)."""
    ps = h.oracle_primes(0, 2)
    for nmax, d, qs in ((1000, 3, [(1000, 2000), (999, 1001)]), (1024, 2, [(1024, 3000), (7, 9)])):
        assert h.emu_residues(ps, nmax, d, qs) == [h.oracle_residues(p, nmax, d, qs) for p in ps]
    p = ps[1]
    assert h.emu_residues([p], 1500, 3, [(1500, 4000), (800, 801)]) == [h.oracle_residues(p, 1500, 3, [(1500, 4000), (800, 801)])]


def test_emulated_kernel_golden_small():
    d, queries, first, count, lines = h.load_fast_golden("fast_small_d3.txt")
    exp = h.expected_by_prime(lines)
    items = sorted(exp.items())[:3]
    primes = [p for (i, p), _ in items]
    got = h.emu_residues(primes, max(n for n, _ in queries), d, queries)
    for ((i, p), want), row in zip(items, got):
        for q, r in zip(queries, row):
            if q in want:
                assert r == want[q], (i, q)


def test_emulated_kernel_32bit_library_primes():
    """The engine accepts any NTT-friendly odd prime: the library CLI's 32-bit ones (config 1)."""
    for rec in h.load_lib_golden():
        if rec[0] == "mod" and rec[2] >= 20:
            _, rep, n, M, d, P, r = rec
            assert h.emu_residues([P], n, d, [(n, M)], rep) == [[r]], rec


def test_emulated_kernel_62bit_primes():
    """Primes below 2^62 select the kernel with [0, 2p) transform values: against the reference's
    -DFP_RB=64 output and the oracle, both models."""
    d, queries, first, count, lines = h.load_fast_golden("fast62_small_d3.txt")
    exp = h.expected_by_prime(lines)
    items = sorted(exp.items())[:2]
    qs = [q for q in queries if q[0] <= 300]
    got = h.emu_residues([p for (i, p), _ in items], 300, d, qs)
    for ((i, p), want), row in zip(items, got):
        for q, r in zip(qs, row):
            if q in want:
                assert r == want[q], (i, q)
    import cuckoo_b200 as cb

    for model in (0, 1):
        ps = cb.prime_range(5, 2, bits=62)
        for nmax, dd, qq in ((64, 2, [(64, 200), (10, 11)]), (1000, 3, [(1000, 1500)])):
            assert h.emu_residues(ps, nmax, dd, qq, model) == [h.oracle_residues(p, nmax, dd, qq, model) for p in ps]


@pytest.mark.parametrize("name", ["fast62_n4096_d2.txt", "fast_n4096_d3.txt"])
def test_emulated_kernel_golden_n4096(name):
    """L = 4096 against the reference's residues, 62-bit and 50-bit primes: chain values and
    transform sums near their bounds occur only at this size and with primes near the top of the
    list (a lazy chain value above 2^62 once broke the 62-bit kernel's Montgomery products)."""
    d, queries, first, count, lines = h.load_fast_golden(name)
    exp = h.expected_by_prime(lines)
    items = sorted(exp.items())[:2]
    qs = [q for q in queries if all(q in want for _, want in items)]
    got = h.emu_residues([p for (i, p), _ in items], max(n for n, _ in qs), d, qs)
    for ((i, p), want), row in zip(items, got):
        assert row == [want[q] for q in qs], (name, i)


@pytest.mark.parametrize("nmax,R", [(1000, 4), (2000, 3), (4000, 3), (4000, 5)])
def test_emulated_tuning_geometries(nmax, R):
    """The autotuner's other register-pass geometries (2^R entries per thread) compute the
    oracle's residues: the same phase code at another thread count and radix."""
    import ctypes

    L = h.emu()
    L.emu_residues_geo.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.emu_residues_geo.restype = ctypes.c_int
    qs = [(nmax, 2 * nmax + 1), (nmax // 3, nmax)]
    J = len(qs)
    qn = (ctypes.c_int * J)(*[q[0] for q in qs])
    qM = (ctypes.c_int * J)(*[q[1] for q in qs])
    pr = (ctypes.c_uint64 * 1)(P0)
    out = (ctypes.c_uint64 * J)()
    assert L.emu_residues_geo(pr, 1, nmax, 3, 0, qn, qM, J, out, R) == 0
    assert [int(x) for x in out] == h.oracle_residues(P0, nmax, 3, qs)


def emu_cluster(primes, nmax, d, queries, lg, C, model=0):
    """The cluster kernel (transform length 2^lg on C CTAs per prime, run as C host threads that
    meet at the cluster barriers and write each other's shared memory) on a table of nmax."""
    import ctypes

    L = h.emu()
    u64, ci = ctypes.c_uint64, ctypes.c_int
    L.emu_residues_cluster.argtypes = [ctypes.POINTER(u64), ci, ci, ci, ci, ctypes.POINTER(ci), ctypes.POINTER(ci), ci,
                                       ctypes.POINTER(u64), ci, ci]
    L.emu_residues_cluster.restype = ci
    B, J = len(primes), len(queries)
    out = (u64 * (B * J))()
    rc = L.emu_residues_cluster((u64 * B)(*primes), B, nmax, d, model, (ci * J)(*[n for n, _ in queries]),
                                (ci * J)(*[M for _, M in queries]), J, out, lg, C)
    assert rc == 0, rc
    return [[int(x) for x in out[b * J:(b + 1) * J]] for b in range(B)]


@pytest.mark.parametrize("lg,C", [(15, 4), (15, 8), (15, -4), (15, -8), (16, 8), (16, 16)])  # -C: 8 entries per thread
@pytest.mark.parametrize("model", [0, 1])
def test_emulated_cluster_kernel_matches_oracle(lg, C, model):
    """Tables above n = 16384 run one prime per cluster of CTAs: pass 0 of each transform on every
    CTA's columns, the exchange through distributed shared memory (with the lazy reduction of the
    forward values the 2^15 and 2^16 bounds need, checked here), the per-CTA powers, row sums and
    flushes, and the first CTA's Horner finish over all CTAs' row sums.  Small tables on the long
    transforms: the residues do not depend on the length."""
    ps = h.oracle_primes(0, 2)
    # rows spread over two or three CTAs (512 or 256 threads each), so every cross-CTA path runs
    nmax, d, qs = (600, 3, [(600, 1500), (513, 1100), (5, 9)]) if model == 0 else (300, 2, [(300, 700), (17, 20)])
    if C == -4:  # 1024 threads per CTA
        nmax, qs = 1100, [(1100, 2500), (1030, 1100)] if model == 0 else [(1100, 2500), (17, 20)]
    assert emu_cluster(ps, nmax, d, qs, lg, C, model) == [h.oracle_residues(p, nmax, d, qs, model) for p in ps]


@pytest.mark.parametrize("lg,C", [(15, 4), (16, 8)])
def test_emulated_cluster_kernel_62bit_primes(lg, C):
    """The cluster kernels for primes below 2^62 (transforms kept in [0, 2p)), at the top of the
    reference's -DFP_RB=64 list, rows over two CTAs."""
    import cuckoo_b200 as cb

    ps = cb.prime_range(0, 2, bits=62)
    nmax, d, qs = 600, 3, [(600, 1500), (513, 1100)]
    assert emu_cluster(ps, nmax, d, qs, lg, C) == [h.oracle_residues(p, nmax, d, qs) for p in ps]
