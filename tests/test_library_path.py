"""The reference's 32-bit library path (`cuckoo_fail single`, config 1 and the replacement model)
on this engine: the library's prime choice through the C ABI, and N_bad recombined from residues
modulo exactly those primes.  CPU tests use the oracle for the residues; the GPU test uses the
engine (cuckoo-failure_b200/single.py)."""
import os
import sys

import pytest

import cuckoo_b200 as cb
import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import crt  # noqa: E402

EXACT = [r for r in h.load_lib_golden() if r[0] == "exact"]


def test_prime_set_of_config_1():
    """What the reference's library CLI prints for n=200, M=400, d=3: 152 primes, from 4276092929
    down to 104857601; 169 with --replacement."""
    ps = cb.lib_primes(200, 400, 3)
    assert len(ps) == 152 and ps[0] == 4276092929 and ps[-1] == 104857601
    assert ps == sorted(ps, reverse=True) and len(set(ps)) == len(ps)
    assert len(cb.lib_primes(200, 400, 3, cb.MODEL_REPLACEMENT)) == 169
    L = cb.transform_length(200)
    assert all(p < 2**32 and (p - 1) % L == 0 for p in ps)


@pytest.mark.parametrize("rec", EXACT, ids=str)
def test_prime_counts_match_library_cli(rec):
    _, rep, n, M, d, nprimes, _, _ = rec
    assert len(cb.lib_primes(n, M, d, rep)) == nprimes


@pytest.mark.parametrize("rec", [r for r in EXACT if r[2] <= 60], ids=str)
def test_library_flow_with_oracle_residues(rec):
    """The same reconstruction as the library, residues from the oracle: N_bad is exact."""
    _, rep, n, M, d, _, _, nbad = rec
    ps = cb.lib_primes(n, M, d, rep)
    x, m = crt.crt([(p, h.oracle_residues(p, n, d, [(n, M)], rep)[0]) for p in ps])
    assert m > crt.q_power(n, M, d, rep == 1) and x == nbad


@pytest.mark.gpu
@pytest.mark.parametrize("rec", EXACT, ids=str)
def test_single_on_gpu_matches_library_cli(rec):
    """Config 1 end to end on the GPU: every residue modulo the library's primes equals the
    oracle's, and the recombined N_bad equals `cuckoo_fail single --exact`."""
    import single

    _, rep, n, M, d, nprimes, pfail, nbad = rec
    with cb.Engine(0) as eng:
        primes, res, x, Qn, _ = single.solve(n, M, d, rep == 1, engine=eng)
    assert len(primes) == nprimes and x == nbad
    for p, r in list(zip(primes, res))[:: max(1, len(primes) // 8)]:
        assert r == h.oracle_residues(p, n, d, [(n, M)], rep)[0]
    if nbad:
        assert x / Qn == pytest.approx(float(pfail), rel=1e-14)
