"""Multi-GPU logic on CPU: two gloo ranks split a prime range (cuckoo-failure_b200/multi.py), each
computes its share (the oracle stands in for the GPU here), rank 0 gathers; the merged output is
byte-identical to the reference's own single-process file.  Also the max-over-ranks timing."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

import helpers as h

sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
import multi  # noqa: E402


def oracle_residues_fn(primes, nmax, d, queries, model):
    return np.array([h.oracle_residues(p, nmax, d, queries, model) for p in primes], dtype=np.uint64)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, d, queries, first, count, out_path):
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(h.ROOT, "cuckoo-failure_b200"))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        f, c = multi.shard(first, count, rank, world)
        recs = multi.rank_lines(d, queries, f, c, oracle_residues_fn)
        merged = multi.gather_to_rank0(recs, dist)
        t = multi.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            with open(out_path, "w") as fo:
                fo.write(multi.format_lines(merged))
                fo.write(f"#max {t}\n")
    finally:
        dist.destroy_process_group()


def test_shard_is_disjoint_and_covering():
    for count in (0, 1, 7, 40, 14184):
        for world in (1, 2, 3, 8):
            got = [multi.shard(5, count, r, world) for r in range(world)]
            idx = [i for f, c in got for i in range(f, f + c)]
            assert idx == list(range(5, 5 + count))


def test_two_gloo_ranks_reproduce_reference_output(tmp_path):
    d, queries, first, count, lines = h.load_fast_golden("fast_small_d3.txt")
    queries = [q for q in queries if q[0] <= 300]  # keep the oracle's share small
    count = 24
    want = "".join(" ".join(map(str, ln)) + "\n" for ln in lines if ln[0] < count and (ln[2], ln[3]) in queries)
    out = tmp_path / "merged.txt"
    mp.start_processes(_rank_main, args=(2, free_port(), d, queries, first, count, str(out)), nprocs=2,
                       join=True, start_method="spawn")
    text = out.read_text()
    body, tail = text[: text.rindex("#max")], text[text.rindex("#max"):]
    assert body == want
    assert tail.strip() == "#max 2.0"
