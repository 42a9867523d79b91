"""Sliding window (lg_snapshot_open_window, lg_store_set_min_level): a window
over levels m..L iterates the full snapshot's edges of levels >= m in the same
order (pinned through the reference's unwindowed iteration), and the tasks
run on it agree with the oracle's windowed restatement."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle
from tests._util import max_rel_err
from tests.test_golden_oracle import window_filter

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12


def _golden_graph(golden):
    hg = HostGraph(int(golden["V"]))
    for lv in golden["levels"]:
        hg.add_level(*lv)
    return hg


def test_golden_windows(golden):
    hg = _golden_graph(golden)
    n = len(golden["levels"])
    with Store() as st:
        st.ingest(hg)
        for l in range(1, n):
            with st.snapshot(l) as full:
                fadj = [full.adjacency(dr, with_edge_ids=True) for dr in (0, 1)]
            for m in range(1, l + 1):
                O = Oracle(int(golden["V"]))
                O.add_levels(golden["levels"])
                O.set_min_level(m)
                with st.snapshot(l, min_level=m) as sn:
                    assert sn.min_level == m
                    for dr in (0, 1):
                        eo, en, ecnt = window_filter(*fadj[dr], m)
                        off, nb = sn.adjacency(dr)
                        assert np.array_equal(off, eo) and np.array_equal(nb, en), (l, m, dr)
                    assert np.array_equal(sn.out_degrees(), O.degrees(l, 0))
                    assert np.array_equal(sn.in_degrees(), O.degrees(l, 1))
                    assert sn.num_edges == int(O.degrees(l, 0).sum())
                    pr = sn.pagerank_pull(int(golden["pr_iters"]), float(golden["damping"]))
                    opr = O.pagerank_pull(l, int(golden["pr_iters"]), float(golden["damping"]))
                    assert max_rel_err(pr, opr) <= PR_TOL, (l, m)
                    for r in golden["roots"]:
                        lv, res = sn.bfs(int(r))
                        ref, reached = O.bfs(l, int(r))
                        assert np.array_equal(lv, ref) and res.reached == reached, (l, m, r)


def test_aging_levels_out():
    spec = workloads.rmat_multiversion(scale=14, seed=8, levels=6, level0=0.6, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    L = hg.num_levels - 1
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(lb.LgError):
                st.set_min_level(2)               # snapshot open
            full = sn.adjacency(0, with_edge_ids=True)
            pr_window = None
        st.set_min_level(2)
        assert st.min_level == 2
        with pytest.raises(lb.LgError):
            st.set_min_level(1)                   # cannot decrease
        with pytest.raises(lb.LgError):
            st.snapshot(1)                        # aged out
        with pytest.raises(lb.LgError):
            st.read_level(0, 0)
        O.set_min_level(2)
        with st.snapshot() as sn:
            assert sn.min_level == 2
            eo, en, _ = window_filter(*full, 2)
            off, nb = sn.adjacency(0)
            assert np.array_equal(off, eo) and np.array_equal(nb, en)
            pr_window = sn.pagerank_pull(10)
            assert max_rel_err(pr_window, O.pagerank_pull(L, 10, 0.85)) <= PR_TOL
            sn.flatten(1)
            assert np.array_equal(sn.pagerank_pull(10), pr_window)
            roots = workloads.pick_roots(sn.out_degrees(), 4, seed=2)
            for r in roots:
                lv, res = sn.bfs(int(r))
                ref, reached = O.bfs(L, int(r))
                assert np.array_equal(lv, ref) and res.reached == reached
        # a new level on top of the window, built on the device
        rng = np.random.default_rng(3)
        src = rng.integers(0, hg.max_nodes, 500).astype(np.uint32)
        dst = rng.integers(0, hg.max_nodes, 500).astype(np.uint32)
        keep = src != dst
        pairs = np.unique(np.stack([src[keep], dst[keep]], 1), axis=0)
        with st.snapshot() as sn:
            live = set()
            off, nb = sn.adjacency(0)
            for s, d in pairs:
                if d in nb[off[s]:off[s + 1]]:
                    live.add((s, d))
        new = np.array([p for p in pairs if (p[0], p[1]) not in live], np.uint32)
        st.build_level(hg.max_nodes, new[:, 0].copy(), new[:, 1].copy())
        O.add_level(new[:, 0].copy(), new[:, 1].copy())
        O.set_min_level(2)
        with st.snapshot() as sn:
            for dr in (0, 1):
                off, nb = sn.adjacency(dr)
                oo, on, _ = O.adjacency(L + 1, dr)
                assert np.array_equal(off, oo) and np.array_equal(nb, on)
        # levels that are aged out stay out; the newest cannot be dropped below
        st.set_min_level(L + 1)
        with pytest.raises(lb.LgError):
            st.drop_level()
