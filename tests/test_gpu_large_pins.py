"""Full-size pins of the CUDA engine, through the C ABI, against the reference's own outputs:

* the replacement model (Q = M^d) at n = 4096 and n = 16384, d = 3, modulo the first primes the
  32-bit library would use itself (`cuckoo_fail single --replacement --mod P`);
* 18 queries (n from 1073 to 16384, M from 1.5 n to 4 n) on one table at n = 16384, d = 3: the
  stage-1-fused query path with several (n_j, M_j), rows q > n_j skipped;
* the first 16 instances of the seeded uneven-batch workload, per d from one table set, at primes
  0, 1 and each instance's last prime;
* resident tables (serving) answering the same 18 queries and the replacement model at n = 16384.
Bit-exact: every residue equals the reference's."""
import os
import sys

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import multi  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = cb.Engine(0)
    yield e
    e.close()


def lib_groups():
    """lib_large records grouped as one batch per (rep, n, M, d): {key: [(P, residue)]}."""
    out = {}
    for rep, n, M, d, P, r in h.load_lib_large():
        out.setdefault((rep, n, M, d), []).append((P, r))
    return out


def test_replacement_model_full_size(eng):
    groups = lib_groups()
    assert (1, 16384, 32768, 3) in groups and (1, 4096, 8192, 3) in groups
    for (rep, n, M, d), items in groups.items():
        got = eng.residues([P for P, _ in items], n, d, [(n, M)], model=rep)
        assert [int(x) for x in got[:, 0]] == [r for _, r in items], (rep, n, M, d)


def test_eighteen_queries_full_size(eng):
    d, queries, first, count, lines = h.load_fast_golden("fast_n16384_d3_J18.txt")
    assert len(queries) == 18 and max(n for n, _ in queries) == 16384
    exp = h.expected_by_prime(lines)
    primes = [p for (i, p) in sorted(exp)]
    got = eng.residues(primes, 16384, d, queries)
    for k, (ip, want) in enumerate(sorted(exp.items())):
        assert {q: int(r) for q, r in zip(queries, got[k])} == want, ip


def test_uneven_sample_per_d_table_sets(eng):
    """Each d's instances share one table per prime, built to the largest n still needing that
    prime (multi.rank_lines, the reference driver's active-query rule)."""
    insts, recs = h.load_uneven_sample()
    fn = lambda ps, nm, dd, qs, m: eng.residues(ps, nm, dd, qs, model=m)
    checked = 0
    for d in sorted({x[2] for x in insts}):
        qs = [(n, M) for n, M, dd in insts if dd == d]
        for i in sorted({r[1] for r in recs if r[0] == d}):
            got = {(n, M): r for _, p, n, M, r in multi.rank_lines(d, qs, i, 1, fn)}
            want = {(n, M): r for dd, ii, p, n, M, r in recs if dd == d and ii == i}
            assert got == want, (d, i)
            checked += len(want)
    assert checked == len(recs)


def test_resident_tables_full_size(eng):
    d, queries, first, count, lines = h.load_fast_golden("fast_n16384_d3_J18.txt")
    exp = h.expected_by_prime(lines)
    primes = [p for (i, p) in sorted(exp)]
    with eng.tables(primes, 16384, max(M for _, M in queries), d) as tab:
        got = tab.query(queries)
    for k, (ip, want) in enumerate(sorted(exp.items())):
        assert {q: int(r) for q, r in zip(queries, got[k])} == want, ip
    items = lib_groups()[(1, 16384, 32768, 3)]
    with eng.tables([P for P, _ in items], 16384, 32768, 3, model=cb.MODEL_REPLACEMENT) as tab:
        got = tab.query([(16384, 32768), (16384, 32768)])
    assert [int(x) for x in got[:, 0]] == [r for _, r in items] == [int(x) for x in got[:, 1]]
