#!/usr/bin/env python3
"""Multi-GPU runs of the batch engine: one process per GPU, each on its own contiguous slice of
the prime range, with no exchange on the data path.  Rank 0 gathers the output lines (host
objects, a few bytes per residue) and writes them in prime order, exactly the lines one
`cuckoo_fast_b200 D QUERIES FIRST COUNT` process would print.

The reference splits a run the same way, by FIRST COUNT per process (fast/README.md:23-25);
this is that split inside one torchrun job:

    torchrun --nproc-per-node 8 --master-addr 127.0.0.1 cuckoo-failure_b200/multi.py D QUERIES FIRST COUNT \\
        [--out FILE] [--replacement]
"""
import argparse
import datetime
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cuckoo_b200 as cb  # noqa: E402


def shard(first, count, rank, world):
    """Rank's contiguous slice (first_r, count_r) of [first, first + count); sizes differ by <= 1."""
    base, extra = divmod(count, world)
    start = first + rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def segments(first, count, needs):
    """Split [first, first + count) where the set of queries with i < need changes:
    [(start, stop, [query indices])] with at least one active query."""
    cuts = sorted({first, first + count} | {k for k in needs if first < k < first + count})
    out = []
    for a, b in zip(cuts, cuts[1:]):
        act = [j for j, k in enumerate(needs) if a < k]
        if act:
            out.append((a, b, act))
    return out


def rank_lines(d, queries, first, count, residues_fn, model=cb.MODEL_SUBSET):
    """Output records (i, p, n, M, residue) for primes first .. first+count-1, in order, only for
    queries with i < need(n, M) (fast/cuckoo_fast.cu:891-898).  residues_fn(primes, nmax, d,
    active_queries, model) returns the [prime][query] residues (the engine, or in tests the oracle)."""
    needs = [cb.need(n, M, d, model) for n, M in queries]
    primes = cb.prime_range(first, count) if count > 0 else []
    out = []
    for a, b, act in segments(first, count, needs):
        qs = [queries[j] for j in act]
        ps = primes[a - first:b - first]
        res = residues_fn(ps, max(n for n, _ in qs), d, qs, model)
        for k, p in enumerate(ps):
            for jj, (n, M) in enumerate(qs):
                out.append((a + k, int(p), n, M, int(res[k][jj])))
    return out


def gather_to_rank0(records, dist):
    """Rank 0 gets every rank's records in prime order (stable within a prime); others get None."""
    if dist is None:
        return records
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, records)
    if dist.get_rank() != 0:
        return None
    merged = [r for part in parts for r in part]
    merged.sort(key=lambda r: r[0])
    return merged


def max_over_ranks(x, dist, device=None):
    """Largest x over all ranks (the job time of a weakly scaled run)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def format_lines(records):
    return "".join(f"{i} {p} {n} {M} {r}\n" for i, p, n, M, r in records)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="multi.py")
    ap.add_argument("d", type=int)
    ap.add_argument("queries")
    ap.add_argument("first", type=int)
    ap.add_argument("count", type=int)
    ap.add_argument("--out")
    ap.add_argument("--replacement", action="store_true")
    a = ap.parse_args(argv)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    model = cb.MODEL_REPLACEMENT if a.replacement else cb.MODEL_SUBSET
    with open(a.queries) as f:
        queries = [tuple(int(x) for x in ln.split()[:2]) for ln in f if len(ln.split()) >= 2]
    torch.cuda.set_device(local)
    dd = None
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
        dd = dist
    first, count = shard(a.first, a.count, rank, world)
    with cb.Engine(local) as eng:
        recs = rank_lines(a.d, queries, first, count,
                          lambda ps, nm, d, qs, m: eng.residues(ps, nm, d, qs, model=m), model)
    merged = gather_to_rank0(recs, dd)
    if merged is not None:
        text = format_lines(merged)
        if a.out:
            with open(a.out, "a") as f:
                f.write(text)
        else:
            sys.stdout.write(text)
    if dd is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
