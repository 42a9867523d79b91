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


def test_pagerank_push_bit_exact(golden):
    """The push restatement adds in vertex order, as the reference's atomic
    adds run on one thread (how the golden vectors were made), so the bits
    match; the pull and push results agree within FP64 rounding."""
    O = build(golden)
    for l in range(len(golden["levels"])):
        pr = O.pagerank_push(l, int(golden["pr_iters"]), float(golden["damping"]))
        assert np.array_equal(pr, golden[f"prpush{l}"]), l
        rel = np.max(np.abs(pr - golden[f"pr{l}"]) / np.abs(golden[f"pr{l}"]))
        assert rel <= 1e-12, (l, rel)


def test_bfs_levels_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        for i, r in enumerate(golden["roots"]):
            lv, reached = O.bfs(l, r)
            assert np.array_equal(lv, golden[f"bfs{l}"][i]), (l, r)
            assert reached == golden[f"bfscount{l}"][i]


def test_sssp_distances_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        for i, r in enumerate(golden["roots"]):
            d, _ = O.sssp(l, r)
            assert np.array_equal(d, golden[f"sssp{l}"][i]), (l, r)


def test_bc_matches_reference_fp32(golden):
    """The reference accumulates BC in FP32; the oracle in FP64."""
    O = build(golden)
    for l in range(len(golden["levels"])):
        bc = O.bc(l, golden["bc_sources"])
        ref = golden[f"bc{l}"].astype(np.float64)
        assert np.all(np.abs(bc - ref) <= 1e-5 * np.maximum(np.abs(bc), 1.0)), l


def test_triangle_count_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        assert O.tc(l) == golden[f"tc{l}"], l


def test_scc_partition_exact(golden):
    O = build(golden)
    for l in range(len(golden["levels"])):
        assert np.array_equal(O.scc(l), golden[f"scc{l}"]), l


def teen_expected(off, nbr, age, K):
    """avg_teen_cnt from the reference's in-adjacency (its own iteration
    order), as avg_teen_cnt.h:96-139 computes it."""
    teen = (age >= 10) & (age < 20)
    cs = np.concatenate([[0], np.cumsum(teen[nbr].astype(np.int64))])
    o = off.astype(np.int64)
    cnt = cs[o[1:]] - cs[o[:-1]]
    sel = age > K
    S, c = int(cnt[sel].sum()), int(sel.sum())
    avg = float(np.float32(S / c)) if c else 0.0
    return cnt.astype(np.int32), avg, S, c


def test_avg_teen_cnt_matches_reference_adjacency(golden):
    O = build(golden)
    V = int(golden["V"])
    rng = np.random.default_rng(21)
    age = rng.integers(0, 60, V).astype(np.int32)
    for l in range(len(golden["levels"])):
        exp = teen_expected(golden[f"adj{l}_1_off"], golden[f"adj{l}_1_nbr"], age, 25)
        avg, cnt, S, c = O.avg_teen_cnt(l, age, 25)
        assert np.array_equal(cnt, exp[0]), l
        assert (avg, S, c) == exp[1:], l


def window_filter(off, nbr, ids, m):
    """Adjacency of a sliding window over levels >= m: the chain ends at the
    first fragment below m, and fragment levels fall along the chain, so this
    is the full iteration restricted to edges whose level is >= m."""
    keep = (ids.astype(np.uint64) >> np.uint64(38)) >= m
    o = off.astype(np.int64)
    cs = np.concatenate([[0], np.cumsum(keep.astype(np.int64))])
    cnt = cs[o[1:]] - cs[o[:-1]]
    return np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint64), nbr[keep], cnt


def test_oracle_window_matches_filtered_reference_iteration(golden):
    for l in range(1, len(golden["levels"])):
        full = build(golden)
        for m in range(1, l + 1):
            O = build(golden)
            O.set_min_level(m)
            for dr in (0, 1):
                off, nb, ids = full.adjacency(l, dr)
                assert np.array_equal(off, golden[f"adj{l}_{dr}_off"])
                eo, en, ecnt = window_filter(off, nb, ids, m)
                wo, wn, _ = O.adjacency(l, dr)
                assert np.array_equal(wo, eo) and np.array_equal(wn, en), (l, m, dr)
                if dr == 0:
                    assert np.array_equal(O.degrees(l, 0), ecnt.astype(np.uint32))


def test_oracle_push_equals_pull_on_windows(golden):
    """On sliding windows too, the push restatement gives the pull vector
    within FP64 rounding (the same sums, added in another order)."""
    iters, d = int(golden["pr_iters"]), float(golden["damping"])
    for l in range(1, len(golden["levels"])):
        for m in range(1, l + 1):
            O = build(golden)
            O.set_min_level(m)
            pull = O.pagerank_pull(l, iters, d)
            push = O.pagerank_push(l, iters, d)
            rel = np.max(np.abs(push - pull) / np.abs(pull))
            assert rel <= 1e-12, (l, m, rel)
