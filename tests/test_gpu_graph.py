"""Graph-captured batches (cf_batch_graph_*): one capture, several replays on a stream, with the
device buffers' contents changed between replays.  Every replay must give the residues of a plain
cf_residues call on the same primes, bit for bit, and the oracle's."""
import numpy as np
import pytest

import cuckoo_b200 as cb
import helpers as h

pytestmark = pytest.mark.gpu


def test_batch_graph_replays_bit_exact():
    import torch

    n, d, queries = 300, 3, [(300, 600), (100, 301)]
    first = cb.prime_range(0, 4)
    second = cb.prime_range(4, 4)
    with cb.Engine(0) as eng:
        dev = torch.device("cuda", 0)
        d_primes = torch.tensor(np.array(first, dtype=np.uint64).view(np.int64), device=dev)
        d_out = torch.zeros(4 * len(queries), dtype=torch.int64, device=dev)
        stream = torch.cuda.Stream(device=dev)
        with eng.batch_graph(d_primes.data_ptr(), 4, n, d, queries, d_out.data_ptr()) as g:
            assert g.launches() == 1
            for primes in (first, first, second):
                with torch.cuda.stream(stream):
                    d_primes.copy_(torch.tensor(np.array(primes, dtype=np.uint64).view(np.int64)).to(dev, non_blocking=False))
                    d_out.zero_()
                g.launch(stream.cuda_stream)
                g.status(stream.cuda_stream)
                got = d_out.cpu().numpy().view(np.uint64).reshape(4, len(queries))
                want = eng.residues(primes, n, d, queries)
                assert np.array_equal(got, want)
                assert [[int(x) for x in row] for row in got] == [h.oracle_residues(p, n, d, queries) for p in primes]
