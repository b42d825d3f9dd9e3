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
                       capture_output=True, text=True, check=True)
    assert r.stdout == golden_text(name)


def test_cli_resume_completes_partial_file(tmp_path):
    d, queries, first, count, _ = h.load_fast_golden("fast_small_d2.txt")
    want = golden_text("fast_small_d2.txt")
    out = tmp_path / "out.txt"
    lines = want.splitlines(keepends=True)
    # keep the first 30 lines, then cut the next prime's lines in half (an interrupted batch)
    out.write_text("".join(lines[:30]))
    r = subprocess.run([cb.CLI_PATH, str(d), write_queries(tmp_path, queries), str(first), str(count), "--out", str(out),
                        "--batch", "7"], capture_output=True, text=True, check=True)
    got = out.read_text().splitlines()
    assert sorted(set(got)) == sorted(set(want.splitlines()))
    # second run: nothing left to do
    r = subprocess.run([cb.CLI_PATH, str(d), write_queries(tmp_path, queries), str(first), str(count), "--out", str(out)],
                       capture_output=True, text=True, check=True)
    assert "nothing to do" in r.stderr
