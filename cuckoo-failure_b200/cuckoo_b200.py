"""Python binding of the B200 engine's C ABI (include/cuckoo_b200.h) through ctypes.

The reference (zcy05331/Cuckoo-Failure) exposes this path as the `cuckoo_fast` CLI
(fast/cuckoo_fast.cu:648-904); this module offers the same operations to Python callers:

    prime_range(first, count)          fixed prime list           (fast/cuckoo_fast.cu:403-432)
    need(n, M, d, model)               primes a query needs      (fast/cuckoo_fast.cu:452-459)
    transform_length(nmax)             NTT length                (fast/cuckoo_fast.cu:460-472)
    Engine(device).residues(...)       one batch of primes       (fast/cuckoo_fast.cu:787-901)

There is no CPU fallback: importing works without a GPU (for the host helpers), but the engine
raises if the CUDA library is missing or no device is present.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libcuckoo_b200.so")
CLI_PATH = os.path.join(PKG, "bin", "cuckoo_fast_b200")

MODEL_SUBSET = 0
MODEL_REPLACEMENT = 1

CF_OK, CF_ERR_ARG, CF_ERR_CUDA, CF_ERR_NOMEM, CF_ERR_UNSUPPORTED, CF_ERR_DEVICE = 0, -1, -2, -3, -4, -5
CF_NOALLOC_SCRATCH_BYTES = 64 << 20  # include/cuckoo_b200.h

_u64p = ctypes.POINTER(ctypes.c_uint64)
_intp = ctypes.POINTER(ctypes.c_int)
_lib = None


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cuckoo_b200 error {code}: {msg}")
        self.code = code


def lib():
    """Load libcuckoo_b200.so (built by cuckoo-failure_b200/build.py); raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python cuckoo-failure_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        L.cf_prime_range.argtypes = [ctypes.c_long, ctypes.c_long, _u64p]
        L.cf_prime_range.restype = ctypes.c_long
        L.cf_need.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cf_need.restype = ctypes.c_long
        L.cf_lib_primes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u64p, ctypes.c_long]
        L.cf_lib_primes.restype = ctypes.c_long
        L.cf_tables_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
        L.cf_tables_bytes.restype = ctypes.c_uint64
        L.cf_tables_build.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.cf_tables_build.restype = ctypes.c_int
        L.cf_tables_query.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _intp, _intp, ctypes.c_int, _u64p]
        L.cf_tables_query.restype = ctypes.c_int
        L.cf_tables_free.argtypes = [ctypes.c_void_p]
        L.cf_tables_free.restype = None
        L.cf_tables_build_async.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.cf_tables_build_async.restype = ctypes.c_int
        L.cf_tables_ready.argtypes = [ctypes.c_void_p]
        L.cf_tables_ready.restype = ctypes.c_int
        L.cf_tables_query_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _intp, _intp, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p]
        L.cf_tables_query_async.restype = ctypes.c_int
        L.cf_engine_set_max_ctas.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_engine_set_max_ctas.restype = ctypes.c_int
        L.cf_engine_set_transform_lg.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_engine_set_transform_lg.restype = ctypes.c_int
        L.cf_resident_primes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cf_resident_primes.restype = ctypes.c_long
        L.cf_tune_variants.argtypes = [ctypes.c_int, _intp, _intp, _intp, ctypes.c_int]
        L.cf_tune_variants.restype = ctypes.c_int
        L.cf_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double), ctypes.c_int, _intp]
        L.cf_autotune.restype = ctypes.c_int
        L.cf_tune_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.cf_tune_set.restype = ctypes.c_int
        L.cf_tune_get.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_tune_get.restype = ctypes.c_int
        L.cf_transform_length.argtypes = [ctypes.c_uint64]
        L.cf_transform_length.restype = ctypes.c_uint64
        L.cf_engine_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.cf_engine_create.restype = ctypes.c_int
        L.cf_engine_destroy.argtypes = [ctypes.c_void_p]
        L.cf_engine_destroy.restype = None
        L.cf_engine_last_error.argtypes = [ctypes.c_void_p]
        L.cf_engine_last_error.restype = ctypes.c_char_p
        L.cf_residues.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  _intp, _intp, ctypes.c_int, _u64p]
        L.cf_residues.restype = ctypes.c_int
        L.cf_residues_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _intp, _intp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.cf_residues_async.restype = ctypes.c_int
        L.cf_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cf_workspace_bytes.restype = ctypes.c_uint64
        L.cf_max_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cf_max_batch.restype = ctypes.c_long
        L.cf_prime_range_bits.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_int, _u64p]
        L.cf_prime_range_bits.restype = ctypes.c_long
        L.cf_need_bits.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cf_need_bits.restype = ctypes.c_long
        L.cf_engine_set_prime_bits.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_engine_set_prime_bits.restype = ctypes.c_int
        L.cf_last_launches.argtypes = [ctypes.c_void_p]
        L.cf_last_launches.restype = ctypes.c_long
        L.cf_batch_graph_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _intp, _intp, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_void_p)]
        L.cf_batch_graph_create.restype = ctypes.c_int
        L.cf_batch_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.cf_batch_graph_launch.restype = ctypes.c_int
        L.cf_batch_graph_status.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.cf_batch_graph_status.restype = ctypes.c_int
        L.cf_batch_graph_launches.argtypes = [ctypes.c_void_p]
        L.cf_batch_graph_launches.restype = ctypes.c_long
        L.cf_batch_graph_destroy.argtypes = [ctypes.c_void_p]
        L.cf_batch_graph_destroy.restype = None
        L.cf_uneven_create.argtypes = [ctypes.c_void_p, _intp, _intp, _intp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.POINTER(ctypes.c_void_p)]
        L.cf_uneven_create.restype = ctypes.c_int
        for f in (L.cf_uneven_outputs, L.cf_uneven_tables, L.cf_uneven_launches):
            f.argtypes = [ctypes.c_void_p]
            f.restype = ctypes.c_long
        L.cf_uneven_offset.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_uneven_offset.restype = ctypes.c_long
        L.cf_uneven_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.cf_uneven_launch.restype = ctypes.c_int
        L.cf_uneven_results.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_void_p]
        L.cf_uneven_results.restype = ctypes.c_int
        L.cf_uneven_destroy.argtypes = [ctypes.c_void_p]
        L.cf_uneven_destroy.restype = None
        L.cf_uneven_describe.argtypes = [_intp, _intp, _intp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                         ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                                         ctypes.c_long]
        L.cf_uneven_describe.restype = ctypes.c_long
        _lib = L
    return _lib


def prime_range(first, count, bits=50):
    """Primes number first .. first+count-1 of the fixed list below 2^bits (bits = 50, or 62 for the
    list of the reference's -DFP_RB=64 build)."""
    out = np.zeros(max(count, 0), dtype=np.uint64)
    got = lib().cf_prime_range_bits(first, count, bits, out.ctypes.data_as(_u64p))
    return [int(x) for x in out[:got]]


def need(n, M, d, model=MODEL_SUBSET, bits=50):
    return int(lib().cf_need_bits(n, M, d, model, bits))


def transform_length(nmax):
    return int(lib().cf_transform_length(nmax))


def lib_primes(n, M, d, model=MODEL_SUBSET):
    """The 32-bit primes of the library CLI for (n, M, d) (src/cuckoo_fail.cpp:151-170)."""
    k = int(lib().cf_lib_primes(n, M, d, model, None, 0))
    if k < 0:
        raise ValueError(f"no prime set for n={n}, M={M}, d={d}")
    out = np.zeros(k, dtype=np.uint64)
    lib().cf_lib_primes(n, M, d, model, out.ctypes.data_as(_u64p), k)
    return [int(x) for x in out]


def tune_variants(lg):
    """The compiled geometries for transform length 2^lg, the default first:
    [{"entries_per_thread": 2^r, "threads": T, "ctas_per_sm": k}]."""
    r, t, m = (np.zeros(8, dtype=np.int32) for _ in range(3))
    k = int(lib().cf_tune_variants(lg, r.ctypes.data_as(_intp), t.ctypes.data_as(_intp), m.ctypes.data_as(_intp), 8))
    return [{"entries_per_thread": 1 << int(r[i]), "threads": int(t[i]), "ctas_per_sm": int(m[i])} for i in range(k)]


def workspace_bytes(nmax, Mmax, J):
    return int(lib().cf_workspace_bytes(nmax, Mmax, J))


def _queries(queries):
    qn = np.ascontiguousarray([q[0] for q in queries], dtype=np.int32)
    qM = np.ascontiguousarray([q[1] for q in queries], dtype=np.int32)
    return qn, qM


class Engine:
    """One CUDA device.  residues() runs one batch of primes through the persistent kernel."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib().cf_engine_create(device, ctypes.byref(h))
        if rc != CF_OK:
            raise EngineError(rc, f"cannot open CUDA device {device}")
        self._h = h

    def close(self):
        if self._h:
            lib().cf_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != CF_OK:
            raise EngineError(rc, lib().cf_engine_last_error(self._h).decode())

    def residues(self, primes, nmax, d, queries, model=MODEL_SUBSET):
        """N_bad(n_j, M_j) mod p for every prime (rows) and query (columns), as a uint64 array."""
        p = np.ascontiguousarray(primes, dtype=np.uint64)
        qn, qM = _queries(queries)
        out = np.zeros((len(p), len(qn)), dtype=np.uint64)
        rc = lib().cf_residues(self._h, p.ctypes.data_as(_u64p), len(p), nmax, d, model, qn.ctypes.data_as(_intp),
                               qM.ctypes.data_as(_intp), len(qn), out.ctypes.data_as(_u64p))
        self._check(rc)
        return out

    def residues_async(self, d_primes_ptr, B, nmax, d, queries, d_out_ptr, stream_ptr=None, model=MODEL_SUBSET):
        """Device-pointer variant (e.g. torch tensors' data_ptr()); enqueued on stream_ptr."""
        qn, qM = _queries(queries)
        rc = lib().cf_residues_async(self._h, ctypes.c_void_p(d_primes_ptr), B, nmax, d, model,
                                     qn.ctypes.data_as(_intp), qM.ctypes.data_as(_intp), len(qn),
                                     ctypes.c_void_p(d_out_ptr), ctypes.c_void_p(stream_ptr or 0))
        self._check(rc)

    def batch_graph(self, d_primes_ptr, B, nmax, d, queries, d_out_ptr, model=MODEL_SUBSET):
        """Capture one batch over device buffers as a CUDA graph (cf_batch_graph_create) for replay."""
        return BatchGraph(self, d_primes_ptr, B, nmax, d, queries, d_out_ptr, model)

    def tables(self, primes, nmax, Fmax, d, model=MODEL_SUBSET):
        """Build and keep the suffix tables of `primes` on the device for later queries."""
        return Tables(self, primes, nmax, Fmax, d, model)

    def uneven(self, instances, model=MODEL_SUBSET, bits=50, first=0, count=-1, stride=1):
        """Plan and capture an uneven batch over instances [(n, M, d)] (cf_uneven_create)."""
        return Uneven(self, instances, model, bits, first, count, stride)

    def tables_async(self, primes, nmax, Fmax, d, model=MODEL_SUBSET, stream_ptr=None):
        """Enqueue the build of resident tables on a stream (cf_tables_build_async); poll ready()."""
        return Tables(self, primes, nmax, Fmax, d, model, stream_ptr=stream_ptr or 0, wait=False)

    def autotune(self, nmax, Mmax, d, B):
        """Time every compiled geometry for nmax's transform length on B primes (cf_autotune) and
        keep the fastest: returns {"lg", "chosen", "rates" (primes/s per geometry), "variants"}."""
        lg = transform_length(nmax).bit_length() - 1
        rates = (ctypes.c_double * 8)()
        chosen = ctypes.c_int(0)
        self._check(lib().cf_autotune(self._h, nmax, Mmax, d, B, rates, 8, ctypes.byref(chosen)))
        vs = tune_variants(lg)
        return {"lg": lg, "chosen": chosen.value, "rates": [rates[i] for i in range(len(vs))], "variants": vs}

    def tune_set(self, lg, variant):
        self._check(lib().cf_tune_set(self._h, lg, variant))

    def tune_get(self, lg):
        return int(lib().cf_tune_get(self._h, lg))

    def resident_primes(self, nmax, Mmax, J=1):
        """Primes one launch runs at the same time (SMs x CTAs per SM, or resident clusters)."""
        return int(lib().cf_resident_primes(self._h, nmax, Mmax, J))

    def set_transform_lg(self, lg):
        """Transforms of at least 2^lg entries (0: the reference's length); residues do not change."""
        self._check(lib().cf_engine_set_transform_lg(self._h, lg))

    def set_max_ctas(self, n):
        """At most n primes (CTAs) per launch of this engine's batches (0: no cap)."""
        self._check(lib().cf_engine_set_max_ctas(self._h, n))

    def max_batch(self, nmax, Mmax, J):
        return int(lib().cf_max_batch(self._h, nmax, Mmax, J))

    def last_launches(self):
        return int(lib().cf_last_launches(self._h))


class BatchGraph:
    """A batch captured once as a CUDA graph with its own workspace; launch() replays it on a stream,
    reading the primes from and writing the residues to the device buffers given at capture."""

    def __init__(self, engine, d_primes_ptr, B, nmax, d, queries, d_out_ptr, model=MODEL_SUBSET):
        qn, qM = _queries(queries)
        h = ctypes.c_void_p()
        rc = lib().cf_batch_graph_create(engine._h, ctypes.c_void_p(d_primes_ptr), B, nmax, d, model,
                                         qn.ctypes.data_as(_intp), qM.ctypes.data_as(_intp), len(qn),
                                         ctypes.c_void_p(d_out_ptr), ctypes.byref(h))
        engine._check(rc)
        self._g = h

    def launch(self, stream_ptr=None):
        rc = lib().cf_batch_graph_launch(self._g, ctypes.c_void_p(stream_ptr or 0))
        if rc != CF_OK:
            raise EngineError(rc, "graph launch failed")

    def status(self, stream_ptr=None):
        """Wait for stream_ptr and raise if the last replay's device checks failed."""
        rc = lib().cf_batch_graph_status(self._g, ctypes.c_void_p(stream_ptr or 0))
        if rc != CF_OK:
            raise EngineError(rc, "graph replay failed its device checks")

    def launches(self):
        """Kernel launches in one replay."""
        return int(lib().cf_batch_graph_launches(self._g))

    def close(self):
        if getattr(self, "_g", None):
            lib().cf_batch_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _instance_arrays(instances):
    n = np.ascontiguousarray([x[0] for x in instances], dtype=np.int32)
    M = np.ascontiguousarray([x[1] for x in instances], dtype=np.int32)
    d = np.ascontiguousarray([x[2] for x in instances], dtype=np.int32)
    return n, M, d


class Uneven:
    """An uneven batch captured as one CUDA graph (one work-queue launch per transform length):
    launch() replays it, results() returns [residues of instance k modulo its primes 0 .. need - 1]."""

    def __init__(self, engine, instances, model=MODEL_SUBSET, bits=50, first=0, count=-1, stride=1):
        self.instances = [tuple(int(v) for v in x) for x in instances]
        n, M, d = _instance_arrays(self.instances)
        h = ctypes.c_void_p()
        rc = lib().cf_uneven_create(engine._h, n.ctypes.data_as(_intp), M.ctypes.data_as(_intp),
                                    d.ctypes.data_as(_intp), len(n), model, bits, first, count, stride, ctypes.byref(h))
        engine._check(rc)
        self._u = h
        self.outputs = int(lib().cf_uneven_outputs(h))
        self.offsets = [int(lib().cf_uneven_offset(h, k)) for k in range(len(n))] + [self.outputs]

    def tables(self):
        return int(lib().cf_uneven_tables(self._u))

    def launches(self):
        return int(lib().cf_uneven_launches(self._u))

    def launch(self, stream_ptr=None):
        rc = lib().cf_uneven_launch(self._u, ctypes.c_void_p(stream_ptr or 0))
        if rc != CF_OK:
            raise EngineError(rc, "uneven batch launch failed")

    def results(self, stream_ptr=None):
        out = np.zeros(max(self.outputs, 1), dtype=np.uint64)
        rc = lib().cf_uneven_results(self._u, out.ctypes.data_as(_u64p), ctypes.c_void_p(stream_ptr or 0))
        if rc != CF_OK:
            raise EngineError(rc, "uneven batch failed its device checks")
        return [out[self.offsets[k]:self.offsets[k + 1]] for k in range(len(self.instances))]

    def close(self):
        if getattr(self, "_u", None):
            lib().cf_uneven_destroy(self._u)
            self._u = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def uneven_describe(instances, model=MODEL_SUBSET, bits=50, first=0, count=-1, stride=1, jcap=0):
    """The plan of an uneven batch without a device: [(d, prime index, lg, n, F, J, q0)] in launch order."""
    n, M, d = _instance_arrays(instances)
    args = (n.ctypes.data_as(_intp), M.ctypes.data_as(_intp), d.ctypes.data_as(_intp), len(n), model, bits, first,
            count, stride, jcap)
    k = int(lib().cf_uneven_describe(*args, None, 0))
    if k < 0:
        raise ValueError("invalid instances")
    buf = (ctypes.c_long * (7 * max(k, 1)))()
    lib().cf_uneven_describe(*args, buf, k)
    return [tuple(buf[7 * t:7 * t + 7]) for t in range(k)]


class Tables:
    """Resident tables of a batch of primes (cf_tables_build); query() answers (n, M) with n <= nmax,
    M <= Fmax from them without a rebuild."""

    def __init__(self, engine, primes, nmax, Fmax, d, model=MODEL_SUBSET, stream_ptr=None, wait=True):
        self.engine, self.nmax, self.Fmax, self.d, self.model = engine, nmax, max(nmax, Fmax), d, model
        self.primes = [int(p) for p in primes]
        p = np.ascontiguousarray(self.primes, dtype=np.uint64)
        h = ctypes.c_void_p()
        if wait:
            rc = lib().cf_tables_build(engine._h, p.ctypes.data_as(_u64p), len(p), nmax, Fmax, d, model, ctypes.byref(h))
        else:
            rc = lib().cf_tables_build_async(engine._h, p.ctypes.data_as(_u64p), len(p), nmax, Fmax, d, model,
                                             ctypes.c_void_p(stream_ptr), ctypes.byref(h))
        engine._check(rc)
        self._t = h

    def ready(self):
        """True once the build has finished; raises if its device checks failed."""
        rc = lib().cf_tables_ready(self._t)
        if rc < 0:
            raise EngineError(rc, "resident table build failed")
        return rc == 1

    def query_async(self, queries, d_out_ptr, stream_ptr=None):
        """Enqueue the residues of `queries` into device memory [prime][query] on a stream."""
        qn, qM = _queries(queries)
        rc = lib().cf_tables_query_async(self.engine._h, self._t, qn.ctypes.data_as(_intp), qM.ctypes.data_as(_intp),
                                         len(qn), ctypes.c_void_p(d_out_ptr), ctypes.c_void_p(stream_ptr or 0))
        self.engine._check(rc)

    def query(self, queries):
        qn, qM = _queries(queries)
        out = np.zeros((len(self.primes), len(qn)), dtype=np.uint64)
        rc = lib().cf_tables_query(self.engine._h, self._t, qn.ctypes.data_as(_intp), qM.ctypes.data_as(_intp),
                                   len(qn), out.ctypes.data_as(_u64p))
        self.engine._check(rc)
        return out

    def close(self):
        if getattr(self, "_t", None):
            lib().cf_tables_free(self._t)
            self._t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def tables_bytes(nmax, Fmax):
    """Device bytes of one prime's resident table."""
    return int(lib().cf_tables_bytes(nmax, Fmax))
