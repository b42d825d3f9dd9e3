"""The CLI (bin/cuckoo_fast_b200) end to end: byte-identical output lines to the reference's
cuckoo_fast for the same arguments, and resume from a partial output file."""
import os
import subprocess

import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu


def golden_text(name):
    with open(os.path.join(h.GOLDEN, name)) as f:
        f.readline()
        return f.read()


def write_queries(tmp_path, queries):
    q = tmp_path / "q.txt"
    q.write_text("".join(f"{n} {M}\n" for n, M in queries))
    return str(q)


@pytest.mark.parametrize("name", ["fast_small_d3.txt", "fast_n300_first17.txt"])
def test_cli_output_identical_to_reference(tmp_path, name):
    d, queries, first, count, _ = h.load_fast_golden(name)
    r = subprocess.run([cb.CLI_PATH, str(d), write_queries(tmp_path, queries), str(first), str(count)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout == golden_text(name)


def run_cli(binary, d, qpath, first, count, out, extra=()):
    r = subprocess.run([binary, str(d), qpath, str(first), str(count), "--out", str(out)] + list(extra),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return r


def test_cli_resume_matches_reference_byte_for_byte(tmp_path):
    """Resume from a file cut inside a prime's lines: the reference redoes every prime whose line
    count is not complete (fast/cuckoo_fast.cu:697-726), so both files must evolve identically."""
    ref_bin = os.path.join(h.ROOT, "oracle", "_ref", "cuckoo_fast_cpu")
    if not os.path.exists(ref_bin):
        pytest.skip("reference host build not available")
    d, queries, first, count, _ = h.load_fast_golden("fast_small_d2.txt")
    qpath = write_queries(tmp_path, queries)
    partial = "".join(golden_text("fast_small_d2.txt").splitlines(keepends=True)[:30])
    mine, ref = tmp_path / "mine.txt", tmp_path / "ref.txt"
    mine.write_text(partial)
    ref.write_text(partial)
    for _ in range(2):
        run_cli(cb.CLI_PATH, d, qpath, first, count, mine, ["--batch", "7"])
        run_cli(ref_bin, d, qpath, first, count, ref)
        assert mine.read_text() == ref.read_text()
    assert set(mine.read_text().splitlines()) == set(golden_text("fast_small_d2.txt").splitlines())


def test_cli_resume_at_prime_boundary(tmp_path):
    d, queries, first, count, lines = h.load_fast_golden("fast_small_d2.txt")
    want = golden_text("fast_small_d2.txt")
    cut = next(k for k, ln in enumerate(lines) if ln[0] == 5)  # first line of prime 5
    out = tmp_path / "out.txt"
    out.write_text("".join(want.splitlines(keepends=True)[:cut]))
    qpath = write_queries(tmp_path, queries)
    run_cli(cb.CLI_PATH, d, qpath, first, count, out, ["--batch", "7"])
    assert out.read_text() == want
    r = run_cli(cb.CLI_PATH, d, qpath, first, count, out)
    assert "nothing to do" in r.stderr


def test_cli_62bit_identical_to_reference_fp_rb_64(tmp_path):
    """--prime-bits 62 against the reference built with -DFP_RB=64, byte for byte."""
    ref_bin = os.path.join(h.ROOT, "oracle", "_ref", "cuckoo_fast_cpu64")
    if not os.path.exists(ref_bin):
        pytest.skip("reference -DFP_RB=64 build not available")
    qpath = write_queries(tmp_path, [(300, 700), (64, 200), (9, 10)])
    mine = subprocess.run([cb.CLI_PATH, "3", qpath, "0", "30", "--prime-bits", "62"], capture_output=True, text=True)
    assert mine.returncode == 0, mine.stderr
    ref = subprocess.run([ref_bin, "3", qpath, "0", "30"], capture_output=True, text=True, check=True)
    assert mine.stdout == ref.stdout
