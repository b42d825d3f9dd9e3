"""Geometry autotuning on the GPU (cf_autotune, cf_tune_*, tune.py): every compiled geometry of a
transform length gives the same residues (the tuner refuses otherwise), the chosen one then runs
the engine's batches and still matches the reference's residues, and the cache round-trips."""
import json

import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_geometry_that_matches_the_reference(tmp_path):
    d, queries, first, count, lines = h.load_fast_golden("fast_n4096_d3.txt")
    exp = h.expected_by_prime(lines)
    with cb.Engine(0) as eng:
        for nmax, B in ((1000, 2 * 148), (4096, 2 * 148)):
            rec = eng.autotune(nmax, 2 * nmax, 3, B)
            assert len(rec["rates"]) == len(cb.tune_variants(rec["lg"])) >= 2
            assert all(r > 0 for r in rec["rates"]) and eng.tune_get(rec["lg"]) == rec["chosen"]
        for k in range(len(cb.tune_variants(12))):  # every n = 4096 geometry against the reference
            eng.tune_set(12, k)
            got = eng.residues([p for (i, p) in sorted(exp)], 4096, d, queries)
            assert [int(r[0]) for r in got] == [exp[ip][queries[0]] for ip in sorted(exp)], k
        with pytest.raises(cb.EngineError):
            eng.tune_set(12, 99)
        import tune

        cache = str(tmp_path / "tune.json")
        a = tune.tuned(eng, 1000, 2000, 3, 148, cache=cache, device_name="test-gpu")
        b = tune.tuned(eng, 1000, 2000, 3, 148, cache=cache, device_name="test-gpu")
        assert a["source"] == "measured" and b["source"] == "cache" and a["chosen"] == b["chosen"]
        assert json.load(open(cache))
