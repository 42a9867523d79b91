"""Pin the CPU oracle (oracle/lgo.cpp) to the reference's own outputs.

tests/golden/*.npz were produced by the reference compiled from source
(tests/golden/make_golden.py).  The oracle restates the reference serially,
so every array, including FP64 PageRank, must match bit for bit.
"""
import numpy as np

from oracle.bind import Oracle


def build(g):
    O = Oracle(int(g["V"]))
    O.add_levels(g["levels"])
    return O


def test_level_arrays_match_reference(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        for dr in (0, 1):
            vt, sl = O.level_arrays(l, dr)
            assert np.array_equal(vt.view(np.uint8), golden[f"vt{l}_{dr}"]), (l, dr)
            assert np.array_equal(sl, golden[f"slots{l}_{dr}"]), (l, dr)


def test_snapshot_iteration_order_matches_reference(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        for dr in (0, 1):
            off, nb, _ = O.adjacency(l, dr)
            assert np.array_equal(off, golden[f"adj{l}_{dr}_off"]), (l, dr)
            assert np.array_equal(nb, golden[f"adj{l}_{dr}_nbr"]), (l, dr)
        assert np.array_equal(O.degrees(l, 0), golden[f"outdeg{l}"])


def test_pagerank_bit_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        pr = O.pagerank_pull(l, int(golden["pr_iters"]), float(golden["damping"]))
        assert np.array_equal(pr, golden[f"pr{l}"]), l


def test_bfs_levels_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        for i, r in enumerate(golden["roots"]):
            lv, reached = O.bfs(l, r)
            assert np.array_equal(lv, golden[f"bfs{l}"][i]), (l, r)
            assert reached == golden[f"bfscount{l}"][i]
