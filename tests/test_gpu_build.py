"""Device-side level construction (lg_store_build_level): levels built on the
GPU from edge deltas are byte-identical to the host builder's levels (which
are byte-identical to the reference's), and snapshots over them agree."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads

pytestmark = pytest.mark.gpu


def _device_ids(vt, slots, level):
    """ids as an ingested level holds them: payloads of this level's
    fragment slots, 0xffffffff elsewhere."""
    ids = np.full(len(slots), 0xffffffff, np.uint32)
    start = vt["adj_list_start"][:-1]
    ln = vt["level_length"][:-1].astype(np.int64)
    own = (start >= 0) & (ln > 0) & ((start.astype(np.uint64) >> np.uint64(38)) == level)
    idx = (start[own].astype(np.uint64) & np.uint64((1 << 38) - 1)).astype(np.int64)
    for i, n in zip(idx, ln[own]):
        ids[i:i + n] = (slots[i:i + n] & np.uint64((1 << 38) - 1)).astype(np.uint32)
    return ids


def _build_all(hg, st, levels=None):
    for l in range(hg.num_levels) if levels is None else levels:
        s, d, ds, dd, w = hg.level_input(l)
        st.build_level(hg.max_nodes, s, d, w, ds, dd)


def _compare_levels(a, b, nlev, weighted):
    for l in range(nlev):
        for dr in (0, 1):
            va, ia = a.read_level(l, dr)
            vb, ib = b.read_level(l, dr)
            assert np.array_equal(va.view(np.uint8), vb.view(np.uint8)), (l, dr)
            assert np.array_equal(ia, ib), (l, dr)
        if weighted:
            _, _, wa = a.read_level(l, 0, weights=True)
            _, _, wb = b.read_level(l, 0, weights=True)
            assert np.array_equal(wa, wb), l


@pytest.mark.parametrize("scale,levels,delete,wmax", [(12, 6, 0.02, 255), (14, 8, 0.005, 0)])
def test_device_built_levels_match_host_builder(scale, levels, delete, wmax):
    spec = workloads.rmat_multiversion(scale=scale, seed=11, levels=levels, level0=0.85,
                                       delete=delete, weight_max=wmax)
    hg = HostGraph.from_spec(spec)
    with Store() as a, Store() as b:
        a.ingest(hg)
        _build_all(hg, b)
        assert b.num_levels == hg.num_levels
        _compare_levels(a, b, hg.num_levels, wmax > 0)
        # the host builder's own arrays
        for l in range(hg.num_levels):
            for dr in (0, 1):
                vt, sl = hg.level_arrays(l, dr)
                vb, ib = b.read_level(l, dr)
                assert np.array_equal(vt.view(np.uint8), vb.view(np.uint8)), (l, dr)
                assert np.array_equal(_device_ids(vt, sl, l), ib), (l, dr)
        for l in range(hg.num_levels):
            with a.snapshot(l) as sa, b.snapshot(l) as sb:
                for dr in (0, 1):
                    oa, na, ea = sa.adjacency(dr, with_edge_ids=True)
                    ob, nb, eb = sb.adjacency(dr, with_edge_ids=True)
                    assert np.array_equal(oa, ob) and np.array_equal(na, nb)
                    assert np.array_equal(ea, eb), (l, dr)
                assert np.array_equal(sa.pagerank_pull(8), sb.pagerank_pull(8))


def test_build_on_top_of_ingested_levels_and_rebuild():
    spec = workloads.rmat_multiversion(scale=13, seed=12, levels=5, level0=0.9,
                                       delete=0.01, weight_max=100)
    hg = HostGraph.from_spec(spec)
    L = hg.num_levels - 1
    with Store() as a, Store() as b:
        a.ingest(hg)
        for l in range(L):
            b.ingest_level(hg.level_desc(l))
        _build_all(hg, b, [L])
        _compare_levels(a, b, hg.num_levels, True)
        # drop and rebuild the newest level: same bytes, same snapshot
        with b.snapshot() as sn:
            pr0 = sn.pagerank_pull(6)
        b.drop_level()
        _build_all(hg, b, [L])
        _compare_levels(a, b, hg.num_levels, True)
        with b.snapshot() as sn:
            assert np.array_equal(sn.pagerank_pull(6), pr0)


def test_build_from_device_tensors():
    import torch
    spec = workloads.rmat_multiversion(scale=12, seed=13, levels=3, level0=0.8, delete=0.02)
    hg = HostGraph.from_spec(spec)
    with Store() as a, Store() as b:
        a.ingest(hg)
        for l in range(hg.num_levels):
            s, d, ds, dd, _ = hg.level_input(l)
            t = [torch.from_numpy(x.astype(np.int32)).cuda() for x in (s, d, ds, dd)]
            b.build_level(hg.max_nodes, t[0], t[1], None, t[2], t[3])
        _compare_levels(a, b, hg.num_levels, False)


def test_build_errors_leave_the_store_unchanged():
    V = 64
    src = np.array([1, 2, 3, 3], np.uint32)
    dst = np.array([2, 3, 4, 5], np.uint32)
    with Store() as st:
        with pytest.raises(lb.LgError):
            st.build_level(V, src, dst, None, [1], [2])            # deletions at level 0
        with pytest.raises(lb.LgError):
            st.build_level(V, [1, 1], [2, 2])                      # duplicate edge
        with pytest.raises(lb.LgError):
            st.build_level(V, [1], [V])                            # id out of range
        assert st.num_levels == 0
        st.build_level(V, src, dst)
        with pytest.raises(lb.LgError):
            st.build_level(V, [7], [8], None, [2], [4])            # (2,4) not live
        with pytest.raises(lb.LgError):
            st.build_level(V, [7], [8], None, [1, 1], [2, 2])      # deleted twice
        with pytest.raises(lb.LgError):
            st.build_level(V, [3], [4])                            # already live
        with pytest.raises(lb.LgError):
            st.build_level(V - 1, [7], [8])                        # max_nodes shrinks
        assert st.num_levels == 1
        st.build_level(V, [3, 9], [9, 1], None, [3], [4])          # delete (3,4), add two
        assert st.num_levels == 2
        with st.snapshot() as sn:
            off, nb = sn.adjacency(0)
            assert list(nb[off[3]:off[4]]) == [9, 5]               # newest fragment first
            assert list(nb[off[1]:off[2]]) == [2]
            assert sn.num_edges == 5
        st.build_level(V, [4], [3], None, [3], [9])                # delete a level-1 edge
        with st.snapshot() as sn:
            off, nb = sn.adjacency(0)
            assert list(nb[off[3]:off[4]]) == [5]
            ioff, inb = sn.adjacency(1)
            assert list(inb[ioff[3]:ioff[4]]) == [4, 2]


def test_build_grows_max_nodes():
    with Store() as st:
        st.build_level(10, [0, 1, 2], [1, 2, 0])
        st.build_level(20, [15, 2], [0, 19], None, [0], [1])
        with st.snapshot(0) as s0:
            assert s0.max_nodes == 10
        with st.snapshot() as sn:
            assert sn.max_nodes == 20
            off, nb = sn.adjacency(0)
            assert list(nb[off[15]:off[16]]) == [0]
            assert list(nb[off[2]:off[3]]) == [19, 0]
            assert list(nb[off[0]:off[1]]) == []
            lv, res = sn.bfs(2)
            assert res.reached == 3 and lv[19] == 1 and lv[0] == 1
