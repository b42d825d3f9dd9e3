"""CRT post-processing (cuckoo-failure_b200/crt.py, the gmpy2-free drop-in for the reference's
fast/post_gmp.py): exact N_bad against the reference's 32-bit library CLI (`cuckoo_fail single
--exact`), the README's known p_fail, and the table built from the reference's own residue files."""
import math
import os
import random
import sys
from fractions import Fraction

import pytest

import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import crt  # noqa: E402

PBITS = 49  # every prime of the engine's fixed list is above 2^49


def residues_50bit(n, M, d, model):
    """Oracle residues of N_bad(n, M) over the first need(n, M) primes of the fixed list."""
    k = crt.need(n, M, d, PBITS, model == 1)
    ps = h.oracle_primes(0, k)
    return [(p, h.oracle_residues(p, n, d, [(n, M)], model)[0]) for p in ps]


@pytest.mark.parametrize("rec", [r for r in h.load_lib_golden() if r[0] == "exact"], ids=str)
def test_exact_nbad_matches_library_cli(rec):
    """N_bad from 50-bit residues equals the library's exact N_bad (computed there from 32-bit
    primes): the integer does not depend on which primes carried it."""
    _, rep, n, M, d, _, pfail, nbad = rec
    x, m = crt.crt(residues_50bit(n, M, d, rep))
    Qn = crt.q_power(n, M, d, rep == 1)
    assert m > 4 * Qn
    assert x == nbad
    if nbad:
        # the library prints p_fail with 16 significant digits from long-double logarithms
        assert float(crt.sci(x, Qn)) == pytest.approx(float(pfail), rel=1e-14)


def test_readme_known_answer():
    """README.md:60-67: cuckoo_fail single -n 20 -M 40 -d 3 gives p_fail = 2.328850077437917e-07."""
    x, _ = crt.crt(residues_50bit(20, 40, 3, 0))
    Qn = crt.q_power(20, 40, 3)
    assert f"{float(Fraction(x, Qn)):.15e}" == "2.328850077437917e-07"  # the README rounds
    assert crt.sci(x, Qn).startswith("2.32885007743791696")  # the table truncates


def test_table_from_reference_residue_file(tmp_path):
    """crt.py over a residue file written by the reference's own fast engine (40 primes): the
    queries covered by 40 primes get complete rows, whose N_bad agrees with an independent prime;
    the others are reported INCOMPLETE."""
    d, queries, first, count, lines = h.load_fast_golden("fast_small_d3.txt")
    path = tmp_path / "out.txt"
    path.write_text("".join(" ".join(map(str, ln)) + "\n" for ln in lines))
    rows = list(crt.table_rows(crt.read_residues([str(path)]), d, PBITS))
    assert rows[0] == crt.HEADER
    body = {(int(r.split("\t")[0]), int(r.split("\t")[1])): r.split("\t") for r in rows[1:]}
    assert sorted(body) == sorted(queries)
    res = crt.read_residues([str(path)])
    complete = 0
    for (n, M), cols in body.items():
        k = crt.need(n, M, d, PBITS)
        assert cols[2] == f"{M / n:.6f}"
        if k > count:
            assert cols[3] == f"INCOMPLETE {count}/{k}"
            continue
        complete += 1
        x, _ = crt.crt([res[(n, M)][i] for i in range(k)])
        Qn = crt.q_power(n, M, d)
        # an independent 32-bit NTT prime that did not take part in the CRT
        P = 998244353
        assert x % P == h.oracle_residues(P, n, d, [(n, M)])[0]
        assert cols[8] == str(k)
        assert cols[7] == crt.sci(x, Qn)
        assert cols[4:7] == ["yes" if (x << lam) <= Qn else "no" for lam in (40, 64, 128)]
    assert complete >= 3


def test_cli_main_writes_table_and_dump(tmp_path, capsys):
    d, queries, first, count, lines = h.load_fast_golden("fast_small_d3.txt")
    path = tmp_path / "out.txt"
    path.write_text("".join(" ".join(map(str, ln)) + "\n" for ln in lines))
    dump = tmp_path / "dump"
    dump.mkdir()
    assert crt.main([str(d), str(path), "--pbits", "49", "--dump", str(dump)]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[0] == crt.HEADER and len(out) == 1 + len(queries)
    files = sorted(os.listdir(dump))
    assert "N_100_150.txt" in files
    text = (dump / "N_100_150.txt").read_text()
    assert text.startswith("N_bad=") and text.endswith("Q^n=C(150,3)^100\n")


def test_sci_is_exact_truncation():
    rng = random.Random(7)
    for _ in range(300):
        N = rng.randrange(1, 10 ** rng.randrange(1, 120))
        D = rng.randrange(1, 10 ** rng.randrange(1, 120))
        s = crt.sci(N, D, digits=40)
        mant, e = s.split("e")
        q = Fraction(N, D)
        # the 40 digits are floor(N / D / 10^(e - 39))
        want = math.floor(q / Fraction(10) ** (int(e) - 39))
        assert mant.replace(".", "") == str(want) and len(str(want)) == 40


def test_log2_column_matches_320_bit_reference():
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 320
    rng = random.Random(11)
    for _ in range(100):
        D = rng.getrandbits(rng.randrange(64, 6000)) | 1
        x = rng.randrange(1, D + 1)
        v = mpmath.log(mpmath.mpf(x), 2) - mpmath.log(mpmath.mpf(D), 2)
        # 15 decimals: the 320-bit value rounded to nearest
        assert Fraction(crt.log2_ratio_text(x, D)) == Fraction(int(mpmath.nint(v * 10**15)), 10**15)
    assert crt.log2_ratio_text(0, 5) == "-inf"


def test_need_matches_post_processing_rule():
    # fast/post_gmp.py:45-47 with --pbits 49 is the engine's need() for the d-subset model
    import cuckoo_b200 as cb

    for n, M, d in ((8, 9, 3), (200, 400, 3), (4096, 8192, 3), (16384, 32768, 2), (16384, 32768, 4)):
        assert crt.need(n, M, d, PBITS) == cb.need(n, M, d)
