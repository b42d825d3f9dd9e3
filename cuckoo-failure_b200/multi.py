#!/usr/bin/env python3
"""Multi-GPU runs of the batch engine: one process per GPU, each on its own contiguous slice of
the prime range, with no exchange on the data path.  Rank 0 gathers the output lines (host
objects, a few bytes per residue) and writes them in prime order, exactly the lines one
`cuckoo_fast_b200 D QUERIES FIRST COUNT` process would print.  With --out the job resumes as the
reference's driver does (fast/cuckoo_fast.cu:697-726): rank 0 reads the file, a prime counts as
done only when every query that needs it has its line there, and only the remaining primes are
split across the ranks and appended.

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


def done_primes(path, needs, first, count):
    """Primes i in [first, first + count) already complete in the output file at `path`: the file
    holds as many lines for i as there are queries with i < need (fast/cuckoo_fast.cu:697-720).
    A prime cut off inside its lines counts as not done (its lines are all written again)."""
    if not path or not os.path.exists(path):
        return set()
    cnt = {}
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if len(t) == 5 and t[0].lstrip("-").isdigit():
                cnt[int(t[0])] = cnt.get(int(t[0]), 0) + 1
    out = set()
    for i in range(first, first + count):
        want = sum(1 for k in needs if i < k)
        if want > 0 and cnt.get(i, 0) == want:
            out.add(i)
    return out


def todo_primes(first, count, needs, done):
    """Prime indices still to compute, in order (fast/cuckoo_fast.cu:722-726)."""
    top = min(first + count, max(needs) if needs else first)
    return [i for i in range(first, top) if i not in done]


def shard_list(todo, rank, world):
    """Rank's contiguous slice of the todo list (sizes differ by at most one)."""
    f, c = shard(0, len(todo), rank, world)
    return todo[f:f + c]


def runs(indices):
    """Maximal runs of consecutive indices: [(first, count)]."""
    out = []
    for i in indices:
        if out and out[-1][0] + out[-1][1] == i:
            out[-1] = (out[-1][0], out[-1][1] + 1)
        else:
            out.append((i, 1))
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


def run_job(d, queries, first, count, residues_fn, out_path=None, dist=None, model=cb.MODEL_SUBSET):
    """One job over all ranks: rank 0 finds the primes still to do (resuming from out_path), every
    rank computes its contiguous share of them, rank 0 gathers and appends the lines to out_path
    (or returns them as text).  Returns the text written on rank 0, None elsewhere."""
    needs = [cb.need(n, M, d, model) for n, M in queries]
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
    todo = [None]
    if rank == 0:
        todo[0] = todo_primes(first, count, needs, done_primes(out_path, needs, first, count))
    if dist:
        dist.broadcast_object_list(todo, src=0)
    recs = []
    for f, c in runs(shard_list(todo[0], rank, world)):
        recs += rank_lines(d, queries, f, c, residues_fn, model)
    merged = gather_to_rank0(recs, dist)
    if merged is None:
        return None
    text = format_lines(merged)
    if out_path:
        with open(out_path, "a") as fo:
            fo.write(text)
    return text


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
    with cb.Engine(local) as eng:
        text = run_job(a.d, queries, a.first, a.count, lambda ps, nm, d, qs, m: eng.residues(ps, nm, d, qs, model=m),
                       a.out, dd, model)
    if text is not None and not a.out:
        sys.stdout.write(text)
    if dd is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
