"""CLI argument handling that exits before any device call (fast/cuckoo_fast.cu:654-695 codes)."""
import subprocess

import cuckoo_b200 as cb


def run(args):
    return subprocess.run([cb.CLI_PATH] + args, capture_output=True, text=True)


def test_cli_usage_and_bad_queries(tmp_path):
    assert run([]).returncode == 2
    q = tmp_path / "q.txt"
    q.write_text("10 10\n")
    assert run(["3", str(q), "0", "5"]).returncode == 2  # M must exceed n
    q.write_text("4 10\n")
    assert run(["3", str(q), "0", "5"]).returncode == 2  # max n below 8
    q.write_text("70000 140000\n")
    assert run(["3", str(q), "0", "5"]).returncode == 2  # beyond this build's table size
    assert run(["3", str(tmp_path / "missing.txt"), "0", "5"]).returncode == 2
    q.write_text("100 200\n")
    assert run(["3", str(q), "0", "5", "--bogus"]).returncode == 2


def test_cli_nothing_to_do_for_complete_file(tmp_path):
    q = tmp_path / "q.txt"
    q.write_text("8 9\n")  # need(8, 9, 3) = 3 primes
    out = tmp_path / "o.txt"
    out.write_text("0 1 8 9 5\n1 1 8 9 5\n2 1 8 9 5\n")
    r = run(["3", str(q), "0", "3", "--out", str(out)])
    assert r.returncode == 0 and "nothing to do" in r.stderr


def test_cli_rejects_bad_prime_bits(tmp_path):
    import subprocess

    import cuckoo_b200 as cb

    q = tmp_path / "q.txt"
    q.write_text("20 40\n")
    r = subprocess.run([cb.CLI_PATH, "3", str(q), "0", "2", "--prime-bits", "40"], capture_output=True, text=True)
    assert r.returncode == 2 and "50 or 62" in r.stderr
