"""PageRank through the entry point that allocates no device memory.

lg_pagerank_pull_noalloc serves callers that must not have the library call
cudaMalloc (for instance a process whose device memory another allocator
already owns, where a new cudaMalloc fails or stalls): it runs on a fixed
scratch area compiled into liblg.so.  Its results must equal those of
lg_pagerank_pull, call after call, although every call reuses the same area.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from llama_b200 import HostGraph, LgError, Store, workloads
from llama_b200._lib import check, lib, ptr

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12


def max_rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), np.finfo(np.float64).tiny)))


def noalloc(snap, iters, damping, out):
    check(lib.lg_pagerank_pull_noalloc(snap.handle, iters, damping, ptr(out)))
    return out


def test_noalloc_matches_pagerank_pull_twice():
    spec = workloads.rmat_multiversion(scale=14, seed=3, levels=4, level0=0.85, delete=0.01)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            ref = sn.pagerank_pull(20, 0.85)
            V = sn.max_nodes
            for _ in range(2):                       # the area keeps the last call's data
                out = noalloc(sn, 20, 0.85, np.empty(V, np.float64))
                assert max_rel(out, ref) <= PR_TOL
            import torch
            dev = torch.empty(V, dtype=torch.float64, device="cuda")
            for _ in range(2):
                noalloc(sn, 20, 0.85, dev)
                st.sync()
                assert max_rel(dev.cpu().numpy(), ref) <= PR_TOL
        with st.snapshot(1) as older:                # another snapshot, same area
            ref1 = older.pagerank_pull(5, 0.9)
            out1 = noalloc(older, 5, 0.9, np.empty(older.max_nodes, np.float64))
            assert max_rel(out1, ref1) <= PR_TOL


def test_noalloc_rejects_graphs_beyond_its_area():
    V = 3_000_000                                    # 24 B per vertex > 64 MiB
    hg = HostGraph(V)
    hg.add_level(np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(LgError) as e:
                noalloc(sn, 3, 0.85, np.empty(V, np.float64))
            assert "scratch" in e.value.message
            ref = sn.pagerank_pull(3, 0.85)          # the allocating call still works
            assert np.isfinite(ref).all()
