"""Shared test helpers: golden fixture parsing, and ctypes bindings of the oracle (the checker)
and of the CPU emulation of the kernel's phase code.  Test infrastructure only."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
EMU_SO = os.path.join(ROOT, "tests", "emu", "libcfemu.so")
EMU_DIR = os.path.join(ROOT, "tests", "emu")
EMU_SRCS = [os.path.join(EMU_DIR, f) for f in ("emu.cpp", "emu_big.cpp", "emu_geo.cpp", "emu_cluster.cpp")]

u64 = ctypes.c_uint64
ci = ctypes.c_int


def build_test_libs():
    """Build the oracle and the emulation harness if missing (plain gcc/g++, seconds)."""
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    csrc = os.path.join(ROOT, "cuckoo-failure_b200", "csrc")
    newest = max(os.path.getmtime(os.path.join(csrc, f)) for f in os.listdir(csrc))
    newest = max([newest, os.path.getmtime(os.path.join(EMU_DIR, "emu_exec.hpp"))] + [os.path.getmtime(f) for f in EMU_SRCS])
    if not os.path.exists(EMU_SO) or os.path.getmtime(EMU_SO) < newest:
        objs = [os.path.splitext(f)[0] + ".o" for f in EMU_SRCS]
        procs = [subprocess.Popen(["g++", "-O2", "-std=c++17", "-fPIC", "-pthread", "-c", f, "-o", o])
                 for f, o in zip(EMU_SRCS, objs)]  # the units compile in parallel
        if any(p.wait() for p in procs):
            raise RuntimeError("the emulation harness did not compile")
        subprocess.run(["g++", "-shared", "-pthread"] + objs + ["-o", EMU_SO], check=True)
        for o in objs:
            os.remove(o)


_oracle = None
_emu = None


def oracle():
    global _oracle
    if _oracle is None:
        build_test_libs()
        L = ctypes.CDLL(ORACLE_SO)
        L.oc_prime_range.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.POINTER(u64)]
        L.oc_prime_range.restype = ctypes.c_long
        L.oc_need.argtypes = [ci, ci, ci, ci]
        L.oc_need.restype = ctypes.c_long
        L.oc_transform_length.argtypes = [u64]
        L.oc_transform_length.restype = u64
        for f in (L.oc_residues_ntt, L.oc_residues_cubic):
            f.argtypes = [u64, ci, ci, ci, ci, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(u64)]
            f.restype = ci
        L.oc_suffix_table.argtypes = [u64, ci, ci, ci, ctypes.POINTER(u64)]
        L.oc_suffix_table.restype = ci
        L.oc_birthday.argtypes = [u64, ci, ci]
        L.oc_birthday.restype = u64
        _oracle = L
    return _oracle


def _qarrays(queries):
    J = len(queries)
    return J, (ci * J)(*[q[0] for q in queries]), (ci * J)(*[q[1] for q in queries])


def oracle_residues(p, nmax, d, queries, model=0, cubic=False):
    J, qn, qM = _qarrays(queries)
    out = (u64 * J)()
    f = oracle().oc_residues_cubic if cubic else oracle().oc_residues_ntt
    rc = f(p, nmax, d, model, J, qn, qM, out)
    assert rc == 0, rc
    return [int(x) for x in out]


def oracle_primes(first, count):
    out = (u64 * count)()
    got = oracle().oc_prime_range(first, count, out)
    return [int(x) for x in out[:got]]


def emu():
    global _emu
    if _emu is None:
        build_test_libs()
        L = ctypes.CDLL(EMU_SO)
        L.emu_residues.argtypes = [ctypes.POINTER(u64), ci, ci, ci, ci, ctypes.POINTER(ci), ctypes.POINTER(ci), ci,
                                   ctypes.POINTER(u64)]
        L.emu_residues.restype = ci
        L.emu_keep_words.argtypes = [ci, ci]
        L.emu_keep_words.restype = ctypes.c_long
        L.emu_keep_build.argtypes = [u64, ci, ci, ci, ci, ctypes.POINTER(u64)]
        L.emu_keep_build.restype = ci
        L.emu_block_cell.argtypes = [ci, ci, ci]
        L.emu_block_cell.restype = ctypes.c_long
        L.emu_block_count.argtypes = [ci]
        L.emu_block_count.restype = ctypes.c_long
        L.emu_block_h.argtypes = [ci]
        L.emu_block_h.restype = ci
        _emu = L
    return _emu


def emu_residues(primes, nmax, d, queries, model=0):
    B = len(primes)
    J, qn, qM = _qarrays(queries)
    pr = (u64 * B)(*primes)
    out = (u64 * (B * J))()
    rc = emu().emu_residues(pr, B, nmax, d, model, qn, qM, J, out)
    assert rc == 0, rc
    return [[int(x) for x in out[b * J:(b + 1) * J]] for b in range(B)]


def load_fast_golden(name):
    """A fixture written by tests/golden/make_golden.py from the reference's cuckoo_fast:
    returns (d, queries, first, count, lines) with lines = [(i, p, n, M, residue)]."""
    with open(os.path.join(GOLDEN, name)) as f:
        head = f.readline()
        lines = [tuple(int(x) for x in ln.split()) for ln in f if ln.strip() and not ln.startswith("#")]
    m = re.match(r"# d=(\d+) queries=(.*) first=(\d+) count=(\d+)", head)
    queries = [tuple(int(x) for x in q.split(",")) for q in m.group(2).split()]
    return int(m.group(1)), queries, int(m.group(3)), int(m.group(4)), lines


def load_lib_golden():
    """tests/golden/lib_cuckoo_fail.txt: ('exact', rep, n, M, d, primes, p_fail, N_bad) and
    ('mod', rep, n, M, d, P, residue) records from the reference's 32-bit library CLI."""
    recs = []
    with open(os.path.join(GOLDEN, "lib_cuckoo_fail.txt")) as f:
        for ln in f:
            if ln.startswith("#") or not ln.strip():
                continue
            t = ln.split()
            if t[0] == "exact":
                recs.append(("exact", int(t[1]), int(t[2]), int(t[3]), int(t[4]), int(t[5]), t[6], int(t[7])))
            else:
                recs.append(("mod", int(t[1]), int(t[2]), int(t[3]), int(t[4]), int(t[5]), int(t[6])))
    return recs


def expected_by_prime(lines):
    """{(i, p): {(n, M): residue}} from golden lines."""
    out = {}
    for i, p, n, M, r in lines:
        out.setdefault((i, p), {})[(n, M)] = r
    return out


def load_lib_large():
    """tests/golden/lib_large.txt: [(rep, n, M, d, P, residue)] from the library CLI's --mod P."""
    out = []
    with open(os.path.join(GOLDEN, "lib_large.txt")) as f:
        for ln in f:
            t = ln.split()
            if t and t[0] == "mod":
                out.append(tuple(int(x) for x in t[1:]))
    return out


def load_uneven_sample():
    """tests/golden/uneven_sample.txt: (instances [(n, M, d)], records [(d, i, p, n, M, residue)])."""
    with open(os.path.join(GOLDEN, "uneven_sample.txt")) as f:
        head = f.readline()
        insts = [tuple(int(x) for x in tok.split(",")) for tok in head.split(":", 1)[1].split()]
        recs = [tuple(int(x) for x in ln.split()) for ln in f if ln.strip() and not ln.startswith("#")]
    return insts, recs
