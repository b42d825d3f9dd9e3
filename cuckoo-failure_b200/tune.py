#!/usr/bin/env python3
"""Autotuning of the kernel geometry with a per-GPU cache.

For a transform length the engine has a few compiled geometries (entries per thread in
registers, threads per prime, CTAs per SM: cuckoo_b200.tune_variants).  `tuned(engine, ...)` returns
the fastest for this GPU model and batch size, from the cache file when it has an entry, else by
timing them all on the device (cf_autotune) and recording the result.  The engine then runs that
geometry for every batch at that length.

    python cuckoo-failure_b200/tune.py --n 4096 --M 8192 --d 3 --batch 592 [--cache FILE]
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cuckoo_b200 as cb  # noqa: E402

DEFAULT_CACHE = os.environ.get("CF_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cuckoo_b200",
                                                                      "tune.json"))


def _key(device_name, lg, B):
    return f"{device_name}|lg={lg}|batch={B}"


def tuned(engine, nmax, Mmax, d, B, cache=DEFAULT_CACHE, device_name=None):
    """The geometry the engine should run for (nmax, B): cached, or measured now and cached.
    Sets it on the engine and returns the record {"lg", "chosen", "rates", "variants", "source"}."""
    if device_name is None:
        import torch

        device_name = torch.cuda.get_device_name(torch.cuda.current_device())
    lg = cb.transform_length(nmax).bit_length() - 1
    key = _key(device_name, lg, B)
    data = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                data = json.load(f)
        except (OSError, ValueError):
            data = {}
    rec = data.get(key)
    if rec is not None and rec.get("variants") == cb.tune_variants(lg):
        engine.tune_set(lg, rec["chosen"])
        return {**rec, "source": "cache"}
    rec = engine.autotune(nmax, Mmax, d, B)
    if cache:
        data[key] = rec
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(data, f, indent=1)
    return {**rec, "source": "measured"}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="tune.py")
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--M", type=int, default=8192)
    ap.add_argument("--d", type=int, default=3)
    ap.add_argument("--batch", type=int, default=592)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--cache", default=DEFAULT_CACHE)
    a = ap.parse_args(argv)
    with cb.Engine(a.device) as eng:
        print(json.dumps(tuned(eng, a.n, a.M, a.d, a.batch, a.cache)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
