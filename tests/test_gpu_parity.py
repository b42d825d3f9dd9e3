"""CUDA engine parity (through the C ABI) against the reference's golden residues and the oracle.
Bit-exact: every residue must equal the reference host build's / the 32-bit library's."""
import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = cb.Engine(0)
    yield e
    e.close()


def check_golden(eng, name, max_primes=None):
    d, queries, first, count, lines = h.load_fast_golden(name)
    exp = h.expected_by_prime(lines)
    items = sorted(exp.items())[:max_primes]
    primes = [p for (i, p), _ in items]
    nmax = max(n for n, _ in queries)
    got = eng.residues(primes, nmax, d, queries)
    n_checked = 0
    for ((i, p), want), row in zip(items, got):
        for q, r in zip(queries, row):
            if q in want:
                assert int(r) == want[q], (name, i, q)
                n_checked += 1
    assert n_checked == sum(len(w) for _, w in items)
    return n_checked


@pytest.mark.parametrize("name", ["fast_small_d2.txt", "fast_small_d3.txt", "fast_small_d4.txt",
                                  "fast_n300_first17.txt", "fast_d1.txt"])
def test_gpu_matches_reference_small(eng, name):
    assert check_golden(eng, name) > 0


def test_gpu_matches_reference_n4096(eng):
    assert check_golden(eng, "fast_n4096_d3.txt") == 4


@pytest.mark.parametrize("name", ["fast_n16384_d2.txt", "fast_n16384_d3.txt", "fast_n16384_d4.txt",
                                  "fast_n16384_d3_first16.txt"])
def test_gpu_matches_reference_n16384(eng, name):
    assert check_golden(eng, name) >= 1


def test_gpu_matches_library_32bit_primes_both_models(eng):
    for rec in h.load_lib_golden():
        if rec[0] != "mod":
            continue
        _, rep, n, M, d, P, r = rec
        assert int(eng.residues([P], n, d, [(n, M)], model=rep)[0, 0]) == r, rec


@pytest.mark.parametrize("model", [0, 1])
def test_gpu_matches_oracle_mixed(eng, model):
    rng = np.random.default_rng(7 + model)
    primes = h.oracle_primes(0, 40)
    for nmax in (9, 31, 100, 513, 1500, 3000):
        d = int(rng.integers(1, 5))
        qs = [(nmax, int(nmax * rng.uniform(1.05, 4)) + 1), (max(1, nmax // 3), nmax + 5)]
        ps = [primes[k] for k in rng.choice(40, 3, replace=False)]
        got = eng.residues(ps, nmax, d, qs, model=model)
        for p, row in zip(ps, got):
            assert [int(x) for x in row] == h.oracle_residues(p, nmax, d, qs, model), (nmax, d, p)


def test_gpu_batch_composition_does_not_change_results(eng):
    primes = h.oracle_primes(0, 300)
    qs = [(700, 1500), (300, 301)]
    full = eng.residues(primes, 700, 3, qs)
    alone = eng.residues(primes[123:124], 700, 3, qs)
    again = eng.residues(primes, 700, 3, qs)
    assert np.array_equal(full[123], alone[0])
    assert np.array_equal(full, again)


def test_gpu_rejects_bad_arguments(eng):
    p0 = h.oracle_primes(0, 1)[0]
    with pytest.raises(cb.EngineError) as e:
        eng.residues([p0 + 2], 100, 3, [(100, 200)])  # not prime / not NTT-friendly
    assert e.value.code == cb.CF_ERR_ARG
    with pytest.raises(cb.EngineError) as e:
        eng.residues([p0], 100, 3, [(101, 200)])  # query beyond the table
    assert e.value.code == cb.CF_ERR_ARG
    with pytest.raises(cb.EngineError) as e:
        eng.residues([p0], 100, 3, [(100, 100)])  # M must exceed n
    assert e.value.code == cb.CF_ERR_ARG
    with pytest.raises(cb.EngineError) as e:
        eng.residues([p0], 65537, 3, [(65537, 140000)])  # above the largest transform length, 2^16
    assert e.value.code == cb.CF_ERR_UNSUPPORTED
    assert eng.residues([], 100, 3, [(100, 200)]).shape == (0, 1)


@pytest.mark.parametrize("name", ["fast62_small_d3.txt", "fast62_n4096_d2.txt", "fast62_n16384_d3.txt"])
def test_gpu_matches_reference_62bit(eng, name):
    """Primes below 2^62 against the reference built with -DFP_RB=64."""
    assert check_golden(eng, name) > 0


def test_gpu_62bit_mixed_with_oracle(eng):
    for model in (0, 1):
        ps = cb.prime_range(40, 3, bits=62)
        qs = [(777, 2000), (100, 101)]
        got = eng.residues(ps, 777, 3, qs, model=model)
        assert [[int(x) for x in r] for r in got] == [h.oracle_residues(p, 777, 3, qs, model) for p in ps]
