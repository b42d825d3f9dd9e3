"""The oracle against the full-size fixtures where it finishes in seconds: the replacement model
at n = 4096 (library --mod P at the library's own primes) and the small instances of the
uneven-batch sample (host build, including each instance's last prime, where only part of its d's
instances are active).  The same fixtures pin the CUDA engine at every size (test_gpu_large_pins)."""
import os
import sys

import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import cuckoo_b200 as cb  # noqa: E402
import uneven  # noqa: E402


def test_fixture_sample_is_the_workload_prefix():
    insts, recs = h.load_uneven_sample()
    assert insts == uneven.instances(len(insts))
    # every instance has its primes 0, 1 and need - 1 pinned
    for n, M, d in insts:
        got = {i for dd, i, p, nn, MM, r in recs if (dd, nn, MM) == (d, n, M)}
        assert {0, 1, cb.need(n, M, d) - 1} <= got, (n, M, d)
    # lines appear exactly for the instances still needing prime i (the reference's active rule)
    for dd, i, p, n, M, r in recs:
        assert i < cb.need(n, M, dd)
        assert p == cb.prime_range(i, 1)[0]


def test_oracle_matches_library_replacement_n4096():
    recs = [r for r in h.load_lib_large() if r[1] == 4096]
    assert len(recs) == 4
    for rep, n, M, d, P, res in recs:
        assert h.oracle_residues(P, n, d, [(n, M)], model=rep)[0] == res, (rep, n, P)


def test_oracle_matches_uneven_sample_small_instances():
    _, recs = h.load_uneven_sample()
    small = [r for r in recs if r[3] <= 2200]
    assert len(small) >= 15
    for d, i, p, n, M, res in small:
        assert h.oracle_residues(p, n, d, [(n, M)])[0] == res, (d, i, n, M)
