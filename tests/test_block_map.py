"""Lifetimes of the folded block map of V / S row storage (block_cell in suffix_engine.cuh, called
through the CPU harness).  Block (P, W), W < P, is written at the flush of tile W and read by the
steps of tile P (row group P); the last row group of V is read again by the finish.  Two blocks
may share a cell only if the earlier one is dead (read in tile P1) by the flush that writes the
later one (flush W2 >= P1), and the pool holds exactly the peak number of live blocks."""
import helpers as h


def check_map(n):
    L = h.emu()
    G = (n - 1) // 16 + 1
    hh = L.emu_block_h(n)
    pool = L.emu_block_count(n)
    assert hh == (G + 1) // 2 and pool == (G - hh) * hh
    cells = {}
    for P in range(G):
        for W in range(P):
            c = L.emu_block_cell(P, W, hh)
            assert 0 <= c < pool, (n, P, W, c)
            cells.setdefault(c, []).append((W, P))
    for c, iv in cells.items():
        iv.sort()
        for (w1, p1), (w2, p2) in zip(iv, iv[1:]):
            assert p1 <= w2 and p1 != G - 1, (n, c, iv)
    peak = max(((k + 1) * (G - 1 - k) for k in range(G)), default=0)
    assert pool == peak


def test_block_map_lifetimes_all_group_counts():
    for G in list(range(1, 200)) + [255, 256, 257, 511, 512, 513, 1023, 1024]:
        check_map(16 * G)
        check_map(16 * G - 7)
