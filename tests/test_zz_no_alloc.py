"""cf_residues_noalloc: the allocation-free entry point, for callers that cannot call cudaMalloc
(their device memory belongs to another allocator, or allocating is not allowed where they run).
It keeps all scratch in a static device array shared by every call, so this file checks it
against the allocating entry point (cf_residues) on two calls in a row: the second call finds
the first call's contents in the array and must still return the same residues.  Collected last
so that a failure here never hides the other tests."""
import ctypes

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu

_u64p = ctypes.POINTER(ctypes.c_uint64)
_intp = ctypes.POINTER(ctypes.c_int)


def noalloc(primes, nmax, d, queries, model=cb.MODEL_SUBSET):
    L = cb.lib()
    f = L.cf_residues_noalloc
    f.argtypes = [_u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _intp, _intp, ctypes.c_int, _u64p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    L.cf_noalloc_last_error.restype = ctypes.c_char_p
    p = np.ascontiguousarray(primes, dtype=np.uint64)
    qn = np.ascontiguousarray([q[0] for q in queries], dtype=np.int32)
    qM = np.ascontiguousarray([q[1] for q in queries], dtype=np.int32)
    out = np.zeros((len(p), len(qn)), dtype=np.uint64)
    rc = f(p.ctypes.data_as(_u64p), len(p), nmax, d, model, qn.ctypes.data_as(_intp), qM.ctypes.data_as(_intp),
           len(qn), out.ctypes.data_as(_u64p), None)
    return rc, out, L.cf_noalloc_last_error().decode()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    cases = [  # the second call reuses the array with a different size and prime set
        (cb.prime_range(0, 20), 1000, 3, [(1000, 2000), (300, 301)], cb.MODEL_SUBSET),
        (cb.prime_range(7, 9), 700, 2, [(700, 1500)], cb.MODEL_REPLACEMENT),
    ]
    with cb.Engine(0) as eng:
        for primes, nmax, d, queries, model in cases:
            want = eng.residues(primes, nmax, d, queries, model=model)
            rc, got, msg = noalloc(primes, nmax, d, queries, model)
            assert rc == cb.CF_OK, msg
            assert np.array_equal(got, want)  # integer residues: exact


def test_noalloc_rejects_tables_beyond_the_scratch():
    rc, _, msg = noalloc(cb.prime_range(0, 1), 8000, 3, [(8000, 16000)])
    assert rc == cb.CF_ERR_NOMEM and "static scratch" in msg


def test_noalloc_matches_reference_fixtures():
    """Pinned directly to the reference's residues (50-bit and 62-bit lists), not only to cf_residues."""
    for name in ("fast_small_d3.txt", "fast_n300_first17.txt", "fast62_small_d3.txt"):
        d, queries, first, count, lines = h.load_fast_golden(name)
        exp = h.expected_by_prime(lines)
        primes = [p for (i, p) in sorted(exp)]
        rc, got, msg = noalloc(primes, max(n for n, _ in queries), d, queries)
        assert rc == cb.CF_OK, msg
        for k, (ip, want) in enumerate(sorted(exp.items())):
            assert {q: int(r) for q, r in zip(queries, got[k]) if q in want} == want, (name, ip)


def largest_fitting_nmax():
    """The largest nmax (one query (nmax, nmax + 1)) whose single-prime scratch layout fits:
    a 256-byte error word, then queries, primes, residues and one workspace, each padded to 256 bytes."""
    words = cb.CF_NOALLOC_SCRATCH_BYTES // 8
    fits = lambda n: 4 * 32 + cb.workspace_bytes(n, n + 1, 1) // 8 <= words
    lo, hi = 16, 16384
    while lo < hi:
        mid = (lo + hi + 1) // 2
        lo, hi = (mid, hi) if fits(mid) else (lo, mid - 1)
    return lo


def test_noalloc_at_the_scratch_limit():
    n = largest_fitting_nmax()
    primes = cb.prime_range(0, 2)
    rc, got, msg = noalloc(primes, n, 3, [(n, n + 1)])
    assert rc == cb.CF_OK, msg  # fits exactly: two launches of one prime each
    with cb.Engine(0) as eng:
        assert np.array_equal(got, eng.residues(primes, n, 3, [(n, n + 1)]))
    rc, _, msg = noalloc(primes[:1], n + 1, 3, [(n + 1, n + 2)])
    assert rc == cb.CF_ERR_NOMEM and "static scratch" in msg, msg
