"""Flat snapshot CSR (lg_snapshot_flatten): PageRank and BFS on a flattened
snapshot give exactly what they give on the level stack, and match the
reference's golden outputs and the oracle."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle
from tests._util import max_rel_err

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12


def _oracle_for(hg):
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    return O


def test_flatten_golden_snapshots(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    iters, d = int(golden["pr_iters"]), float(golden["damping"])
    with Store() as st:
        st.ingest(hg)
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                pr0 = sn.pagerank_pull(iters, d)
                assert not sn.is_flat(0) and not sn.is_flat(1)
                sn.flatten(1)
                assert sn.is_flat(1) and not sn.is_flat(0)
                assert np.array_equal(sn.pagerank_pull(iters, d), pr0), l   # same kernels, same bits
                assert max_rel_err(pr0, golden[f"pr{l}"]) <= PR_TOL, l
                sn.flatten(0)
                sn.flatten(0)                                   # already flat: no-op
                for i, r in enumerate(golden["roots"]):
                    lv, res = sn.bfs(int(r))
                    assert np.array_equal(lv, golden[f"bfs{l}"][i]), (l, r)
                    assert res.reached == golden[f"bfscount{l}"][i]
                sn.unflatten()
                assert not sn.is_flat(1)
                assert np.array_equal(sn.pagerank_pull(iters, d), pr0)


@pytest.mark.parametrize("flat_dirs", [(1,), (0,), (0, 1)])
def test_flatten_multiversion_vs_oracle(flat_dirs):
    spec = workloads.rmat_multiversion(scale=15, seed=2, levels=8, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        for l in (0, 3, 7):
            with st.snapshot(l) as sn:
                roots = workloads.pick_roots(sn.out_degrees(), 6, seed=l)
                plain_pr = sn.pagerank_pull(12, 0.85)
                plain_bfs = [sn.bfs(int(r)) for r in roots]
                for dr in flat_dirs:
                    sn.flatten(dr)
                pr = sn.pagerank_pull(12, 0.85)
                assert np.array_equal(pr, plain_pr)
                assert max_rel_err(pr, O.pagerank_pull(l, 12, 0.85)) <= PR_TOL
                for r, (plv, pres) in zip(roots, plain_bfs):
                    lv, res = sn.bfs(int(r))
                    ref, reached = O.bfs(l, int(r))
                    assert np.array_equal(lv, ref), (l, r)
                    assert np.array_equal(lv, plv)
                    assert res.reached == reached == pres.reached
                    assert res.reach_edges == pres.reach_edges


def test_flatten_large_hubs_cross_tiles():
    """Scale 17, one level: in-hubs span many 256-edge tiles and rows of every
    length meet tile boundaries."""
    spec = workloads.rmat_single_level(scale=17, seed=3)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            assert np.max(sn.in_degrees()) > 256 * 30
            sn.flatten(1)
            pr = sn.pagerank_pull(10, 0.85)
            assert max_rel_err(pr, O.pagerank_pull(0, 10, 0.85)) <= PR_TOL
            lv, res = sn.bfs(0)
            ref, reached = O.bfs(0, 0)
            assert np.array_equal(lv, ref) and res.reached == reached


def test_flatten_edgeless_and_all_deleted():
    """A level with no edges, then one that deletes every edge: rows without
    in-edges only."""
    V = 300
    rng = np.random.default_rng(9)
    src = rng.integers(0, V, 900).astype(np.uint32)
    dst = rng.integers(0, V, 900).astype(np.uint32)
    keep = src != dst
    pairs = np.unique(np.stack([src[keep], dst[keep]], 1), axis=0)
    hg = HostGraph(V)
    hg.add_level(pairs[:, 0].copy(), pairs[:, 1].copy())
    hg.add_level(np.empty(0, np.uint32), np.empty(0, np.uint32),
                 pairs[:, 0].copy(), pairs[:, 1].copy())
    with Store() as st:
        st.ingest(hg)
        with st.snapshot(1) as sn:
            assert sn.num_edges == 0
            sn.flatten(0)
            sn.flatten(1)
            pr = sn.pagerank_pull(5, 0.85)
            assert np.all(pr == (1.0 - 0.85) / V)
            lv, res = sn.bfs(7)
            assert res.reached == 1 and lv[7] == 0
            assert np.all(np.delete(lv, 7) == lb.LG_UNREACHED)
            pr0 = sn.pagerank_pull(0, 0.85)
            assert np.all(pr0 == 1.0 / V)


def test_flatten_errors():
    spec = workloads.rmat_single_level(scale=10, seed=1)
    hg = HostGraph.from_spec(spec, reverse_edges=False)
    with Store(reverse_edges=False) as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(lb.LgError):
                sn.flatten(1)                  # no in-CSR
            with pytest.raises(lb.LgError):
                sn.flatten(2)
            sn.flatten(0)
            assert sn.is_flat(0)
            lv, res = sn.bfs(0)                # top-down only, on the flat out-CSR
            assert lv[0] == 0


def test_gather_pass_checksum_and_state():
    """lg_pagerank_gather_pass gathers pr0 / out_degree(src) once per live
    in-edge of the flat in-CSR; it needs the snapshot flattened."""
    from llama_b200 import LgError
    spec = workloads.rmat_multiversion(scale=12, seed=5, levels=3, level0=0.9, delete=0.02)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(LgError):
                sn.gather_pass()
            sn.flatten(1)
            got = sn.gather_pass()
            assert sn.gather_pass(3) == got            # every pass gathers the same
            off, nb = sn.adjacency(1)
            od = sn.out_degrees().astype(np.float64)
            want = float(np.sum((1.0 / sn.max_nodes) / od[nb]))
            assert abs(got - want) <= 1e-12 * abs(want)
