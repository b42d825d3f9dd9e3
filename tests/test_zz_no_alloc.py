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
