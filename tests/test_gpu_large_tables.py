"""Tables above n = 16384 (transform lengths 2^15 and 2^16, one prime per thread-block cluster of
CTAs) through the C ABI: against the reference host build's residues at n = 32768 and n = 65536
(tests/golden, made by make_golden.py --groups huge), through the CLI, and against the oracle on
small tables run on the long transforms with every compiled cluster size.  Bit-exact."""
import os
import subprocess
import tempfile

import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu

CLI = os.path.join(h.ROOT, "cuckoo-failure_b200", "bin", "cuckoo_fast_b200")


@pytest.mark.parametrize("lg,variant", [(15, 0), (15, 1), (15, 2), (15, 3), (16, 0), (16, 1)])
@pytest.mark.parametrize("model", [0, 1])
def test_cluster_kernels_match_oracle_on_small_tables(lg, variant, model):
    ps = cb.prime_range(0, 3)
    # rows spread over two or three CTAs of the cluster (512 or 256 threads each)
    nmax, d, qs = (1300, 3, [(1300, 2700), (1030, 2100), (513, 1100), (7, 9)]) if model == 0 else (1100, 2, [(1100, 2300), (64, 65)])
    with cb.Engine(0) as eng:
        eng.set_transform_lg(lg)
        eng.tune_set(lg, variant)
        assert eng.tune_get(lg) == variant
        got = eng.residues(ps, nmax, d, qs, model=model)
    for p, row in zip(ps, got):
        assert [int(x) for x in row] == h.oracle_residues(p, nmax, d, qs, model), (lg, variant, p)


@pytest.mark.parametrize("name", ["fast_n32768_d3.txt", "fast_n65536_d3.txt", "fast62_n32768_d3.txt",
                                  "fast_n65536_d3_J126.txt"])
def test_large_tables_match_reference(name):
    d, queries, first, count, lines = h.load_fast_golden(name)
    exp = h.expected_by_prime(lines)
    primes = [p for (i, p) in sorted(exp)]
    nmax = max(n for n, _ in queries)
    with cb.Engine(0) as eng:
        got = eng.residues(primes, nmax, d, queries)
    for ((i, p), want), row in zip(sorted(exp.items()), got):
        assert {q: int(r) for q, r in zip(queries, row)} == want, (name, i)


def test_cli_at_n32768_prints_the_reference_lines():
    d, queries, first, count, lines = h.load_fast_golden("fast_n32768_d3.txt")
    with tempfile.TemporaryDirectory() as tmp:
        q = os.path.join(tmp, "q.txt")
        with open(q, "w") as f:
            f.write("".join(f"{n} {M}\n" for n, M in queries))
        out = subprocess.run([CLI, str(d), q, "0", "2"], check=True, capture_output=True, text=True).stdout
    assert sorted(tuple(int(x) for x in ln.split()) for ln in out.splitlines()) == sorted(lines)


def test_large_tables_refuse_what_they_do_not_cover():
    with cb.Engine(0) as eng:
        with pytest.raises(cb.EngineError):  # beyond 2^16
            eng.residues(cb.prime_range(0, 1), 70000, 3, [(70000, 140000)])
        with pytest.raises(cb.EngineError):  # resident tables stop at 16384
            eng.tables(cb.prime_range(0, 1), 20000, 40000, 3)


@pytest.mark.parametrize("lg", [15, 16])
def test_62bit_cluster_kernels_match_oracle_on_small_tables(lg):
    ps = cb.prime_range(0, 2, bits=62)
    nmax, d, qs = 700, 3, [(700, 1500), (513, 1100), (7, 9)]
    with cb.Engine(0) as eng:
        eng.set_transform_lg(lg)
        got = eng.residues(ps, nmax, d, qs)
    for p, row in zip(ps, got):
        assert [int(x) for x in row] == h.oracle_residues(p, nmax, d, qs), (lg, p)


def test_resident_primes_gives_whole_waves():
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    with cb.Engine(0) as eng:
        one = eng.resident_primes(16384, 32768)  # one CTA of 1024 threads per SM
        cl4 = eng.resident_primes(32768, 65536)  # clusters of 4 CTAs, one per SM
        cl8 = eng.resident_primes(65536, 131072)  # clusters of 8
    assert one == sms
    assert 0 < 4 * cl4 <= sms and 0 < 8 * cl8 <= sms
