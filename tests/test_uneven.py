"""Uneven batches (many (n, M, d) instances, each modulo its own need(n, M, d) primes) through one
graph of work-queue launches (cf_uneven_*).

CPU: the C planner equals the restated reference rule (per d and prime, the instances still
needing the prime, one table at their largest n), ordered heaviest first, with query splitting;
the kernel's per-table code run in the CPU harness (own n, F and queries per table, each in a
poisoned slot laid out for its length group, residues scattered by output index) equals the
oracle per instance.
GPU: the graph's residues equal each instance's plain run and the reference's sampled residues;
one kernel launch per transform length."""
import ctypes
import os
import sys

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import multi  # noqa: E402
import uneven  # noqa: E402


def small_instances(seed, count, n_lo, n_hi):
    return uneven.instances(count, seed=seed, n_lo=n_lo, n_hi=n_hi)


def test_plan_is_the_reference_rule():
    for seed, (lo, hi), kw in ((1, (8, 700), {}), (2, (256, 16384), {"stride": 97}),
                               (3, (64, 3000), {"first": 40, "count": 300, "stride": 7})):
        insts = small_instances(seed, 40, lo, hi)
        want = uneven.tables(insts, cb.need, **kw)
        got = cb.uneven_describe(insts, **kw)
        assert len(got) == len(want)
        keys = [(d, i) for d, i, *_ in got]
        assert set(keys) == set(want)
        for d, i, lg, n, F, J, q0 in got:
            act = want[(d, i)]
            assert J == len(act) and n == max(insts[k][0] for k in act)
            assert F == max([n] + [insts[k][1] for k in act])
            assert 1 << lg == cb.transform_length(n)
        # heaviest first: transform length, then table size, then queries
        weights = [(lg, n, J) for _, _, lg, n, _, J, _ in got]
        assert weights == sorted(weights, reverse=True)


def test_plan_splits_tables_beyond_the_query_cap():
    insts = small_instances(4, 30, 100, 400)
    whole = cb.uneven_describe(insts)
    split = cb.uneven_describe(insts, jcap=4)
    assert max(J for *_, J, _ in split) <= 4
    per = {}
    for d, i, lg, n, F, J, q0 in split:
        per[(d, i)] = per.get((d, i), 0) + J
    assert per == {(d, i): J for d, i, lg, n, F, J, q0 in whole}


def emu_uneven(insts, model=0, bits=50, first=0, count=-1, stride=1):
    L = h.emu()
    L.emu_uneven.argtypes = [ctypes.POINTER(ctypes.c_int)] * 3 + [ctypes.c_int] * 3 + [ctypes.c_long] * 3 + [
        ctypes.POINTER(ctypes.c_uint64)]
    L.emu_uneven.restype = ctypes.c_int
    n = (ctypes.c_int * len(insts))(*[x[0] for x in insts])
    M = (ctypes.c_int * len(insts))(*[x[1] for x in insts])
    d = (ctypes.c_int * len(insts))(*[x[2] for x in insts])
    needs = [cb.need(a, b, c, model, bits) for a, b, c in insts]
    out = (ctypes.c_uint64 * sum(needs))()
    assert L.emu_uneven(n, M, d, len(insts), model, bits, first, count, stride, out) == 0
    res, at = [], 0
    for k in needs:
        res.append([int(x) for x in out[at:at + k]])
        at += k
    return res


def test_emulated_queue_equals_oracle_per_instance():
    insts = small_instances(5, 10, 8, 200)
    res = emu_uneven(insts, stride=3)
    for (n, M, d), r in zip(insts, res):
        ps = cb.prime_range(0, cb.need(n, M, d))
        for i in range(0, len(ps), 3):
            assert r[i] == h.oracle_residues(ps[i], n, d, [(n, M)])[0], (n, M, d, i)
        assert all(r[i] == 0 for i in range(len(ps)) if i % 3)  # primes left out of the plan


def test_emulated_queue_replacement_model():
    insts = [(30, 45, 2), (17, 60, 3), (40, 41, 2)]
    res = emu_uneven(insts, model=cb.MODEL_REPLACEMENT, stride=5)
    for (n, M, d), r in zip(insts, res):
        ps = cb.prime_range(0, cb.need(n, M, d, cb.MODEL_REPLACEMENT))
        for i in range(0, len(ps), 5):
            assert r[i] == h.oracle_residues(ps[i], n, d, [(n, M)], cb.MODEL_REPLACEMENT)[0]


def test_uneven_mix_equals_alone_with_oracle():
    """multi.rank_lines (one launch per run of primes with one query set) on the oracle."""
    insts = small_instances(4, 8, 8, 40)
    recs = {}
    for d in sorted({x[2] for x in insts}):
        qs = sorted({(n, M) for n, M, dd in insts if dd == d})
        count = max(cb.need(n, M, d) for n, M in qs)
        fn = lambda primes, nmax, dd, queries, model: np.array(
            [h.oracle_residues(p, nmax, dd, queries, model) for p in primes], dtype=np.uint64)
        for i, p, n, M, r in multi.rank_lines(d, qs, 0, count, fn):
            recs[(d, n, M, i)] = r
    for n, M, d in insts:
        for i, p in enumerate(cb.prime_range(0, cb.need(n, M, d))):
            assert recs[(d, n, M, i)] == h.oracle_residues(p, n, d, [(n, M)])[0]


@pytest.mark.gpu
def test_uneven_graph_equals_each_instance_alone():
    insts = small_instances(7, 24, 16, 700)
    with cb.Engine(0) as eng:
        with eng.uneven(insts) as u:
            lgs = {lg for _, _, lg, *_ in cb.uneven_describe(insts)}
            assert u.launches() == len(lgs)
            u.launch()
            got = u.results()
            u.launch()  # a replay gives the same residues
            again = u.results()
        alone = uneven.per_instance(eng, insts, cb.prime_range, cb.need)
    for k, (n, M, d) in enumerate(insts):
        assert [int(x) for x in got[k]] == alone[k] == [int(x) for x in again[k]], (n, M, d)


@pytest.mark.gpu
def test_uneven_graph_matches_reference_sample():
    """The first 16 instances of the uneven-batch workload against the reference's residues at
    primes 0, 1 and each instance's last prime: each of those prime sets planned on its own."""
    insts, recs = h.load_uneven_sample()
    want = {(d, i, n, M): r for d, i, p, n, M, r in recs}
    points = sorted({i for _, i, *_ in recs} - {1})  # primes 0 and 1 are one plan
    checked = 0
    with cb.Engine(0) as eng:
        for i in points:
            res = uneven.run(eng, insts, first=i, count=2 if i == 0 else 1)
            for (n, M, d), r in zip(insts, res):
                for ii in ((0, 1) if i == 0 else (i,)):
                    if (d, ii, n, M) in want:
                        assert int(r[ii]) == want[(d, ii, n, M)], (n, M, d, ii)
                        checked += 1
    assert checked == len(recs)
