"""Host output mode LG_OUTPUT_ASYNC (lg_store_set_output_mode): results copied
to page-locked host tensors on the store's copy stream equal the ones returned
synchronously, including when more outputs are queued than there are staging
slots; pageable and small outputs stay synchronous."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads

pytestmark = pytest.mark.gpu


def _store_and_roots(scale):
    spec = workloads.rmat_multiversion(scale=scale, seed=4, levels=3, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    st = Store()
    st.ingest(hg)
    return hg, st


def test_async_outputs_match_sync():
    import torch
    hg, st = _store_and_roots(scale=17)
    V = hg.max_nodes
    with st:
        with st.snapshot() as sn:
            roots = workloads.pick_roots(sn.out_degrees(), 6, seed=1)
            ref_lv, ref_rs = sn.bfs_multi(roots)
            ref_pr = sn.pagerank_pull(10, 0.85)
            ref_pr2 = sn.pagerank_pull(3, 0.85)
            st.set_output_mode("async")
            lv = torch.full((len(roots), V), -7, dtype=torch.int32).pin_memory()
            pr = torch.zeros(V, dtype=torch.float64).pin_memory()
            pr2 = torch.zeros(V, dtype=torch.float64).pin_memory()
            assert pr.numel() * 8 >= lb._lib.LG_ASYNC_MIN_BYTES
            # three large outputs in flight with two staging slots
            sn.flatten(1)
            _, rs = sn.bfs_multi(roots, out=lv)
            sn.pagerank_pull(10, 0.85, out=pr)
            sn.pagerank_pull(3, 0.85, out=pr2)
            st.sync()
            assert np.array_equal(lv.numpy(), ref_lv)
            assert [(r.reached, r.reach_edges) for r in rs] == \
                [(r.reached, r.reach_edges) for r in ref_rs]
            assert np.array_equal(pr.numpy(), ref_pr)
            assert np.array_equal(pr2.numpy(), ref_pr2)
            # pageable outputs are returned synchronously in either mode
            assert np.array_equal(sn.pagerank_pull(10, 0.85), ref_pr)
            st.set_output_mode("sync")
            pr.zero_()
            sn.pagerank_pull(10, 0.85, out=pr)
            assert np.array_equal(pr.numpy(), ref_pr)


def test_async_small_output_is_synchronous():
    import torch
    hg, st = _store_and_roots(scale=12)
    V = hg.max_nodes
    assert V * 8 < lb._lib.LG_ASYNC_MIN_BYTES
    with st:
        st.set_output_mode("async")
        with st.snapshot() as sn:
            ref = sn.pagerank_pull(5, 0.85)
            pr = torch.zeros(V, dtype=torch.float64).pin_memory()
            sn.pagerank_pull(5, 0.85, out=pr)
            assert np.array_equal(pr.numpy(), ref)      # no sync needed


def test_output_mode_rejects_unknown():
    _, st = _store_and_roots(scale=10)
    with st:
        with pytest.raises(lb.LgError):
            st.set_output_mode(7)
