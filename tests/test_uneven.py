"""Uneven batch (config 4 pattern): instances with different (n, M) and d, each modulo its own
need(n, M, d) primes.  Per d, one launch per prime segment evaluates every instance that still
needs those primes (the reference driver's active-query rule, fast/cuckoo_fast.cu:789-792);
each instance's residues must equal its own one-instance run."""
import os
import sys

import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import multi  # noqa: E402


def instances(seed, count, n_lo, n_hi):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        out.append((n, n * int(rng.choice([2, 3, 4])), int(rng.choice([2, 3, 4]))))
    return out


def mixed_records(insts, residues_fn):
    recs = {}
    for d in sorted({x[2] for x in insts}):
        qs = sorted({(n, M) for n, M, dd in insts if dd == d})
        count = max(cb.need(n, M, d) for n, M in qs)
        for i, p, n, M, r in multi.rank_lines(d, qs, 0, count, residues_fn):
            recs[(d, n, M, i)] = r
    return recs


def oracle_fn(primes, nmax, d, queries, model):
    return np.array([h.oracle_residues(p, nmax, d, queries, model) for p in primes], dtype=np.uint64)


def test_uneven_mix_equals_alone_with_oracle():
    insts = instances(4, 8, 8, 40)
    recs = mixed_records(insts, oracle_fn)
    for n, M, d in insts:
        for i, p in enumerate(cb.prime_range(0, cb.need(n, M, d))):
            assert recs[(d, n, M, i)] == h.oracle_residues(p, n, d, [(n, M)])[0]


@pytest.mark.gpu
def test_uneven_mix_equals_alone_on_gpu():
    insts = instances(7, 24, 16, 700)
    with cb.Engine(0) as eng:
        fn = lambda ps, nm, d, qs, m: eng.residues(ps, nm, d, qs, model=m)
        recs = mixed_records(insts, fn)
        for n, M, d in insts:
            ps = cb.prime_range(0, cb.need(n, M, d))
            alone = eng.residues(ps, n, d, [(n, M)])[:, 0]
            assert [recs[(d, n, M, i)] for i in range(len(ps))] == [int(x) for x in alone], (n, M, d)
