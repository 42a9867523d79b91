"""PageRank push (lg_pagerank_push, task pagerank_double_push) on the GPU
against the reference's push vectors (golden fixtures), the oracle, and the
pull variant: FP64 within 1e-12 (the atomic adds run in any order)."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle
from tests._util import max_rel_err

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12


def test_golden_push(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    iters, d = int(golden["pr_iters"]), float(golden["damping"])
    with Store() as st:
        st.ingest(hg)
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                for flat in (False, True):
                    if flat:
                        sn.flatten(0)           # scatter over the flat out-CSR
                    pr = sn.pagerank_push(iters, d)
                    assert max_rel_err(pr, golden[f"prpush{l}"]) <= PR_TOL, (l, flat)
                    assert max_rel_err(pr, golden[f"pr{l}"]) <= PR_TOL, (l, flat)


def test_push_multiversion_vs_oracle():
    spec = workloads.rmat_multiversion(scale=15, seed=3, levels=6, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    with Store() as st:
        st.ingest(hg)
        for l in (0, 5):
            with st.snapshot(l) as sn:
                pr = sn.pagerank_push(15, 0.85)
                assert max_rel_err(pr, O.pagerank_push(l, 15, 0.85)) <= PR_TOL
                assert max_rel_err(pr, sn.pagerank_pull(15, 0.85)) <= PR_TOL


def test_push_without_reverse_edges():
    """A store kept without the in-CSR cannot run the pull variant; push
    needs only the out-edges."""
    spec = workloads.rmat_single_level(scale=12, seed=4)
    hg = HostGraph.from_spec(spec, reverse_edges=False)
    O = Oracle(hg.max_nodes)
    O.add_level(*hg.level_input(0)[:4])
    with Store(reverse_edges=False) as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(lb.LgError):
                sn.pagerank_pull(10, 0.85)
            pr = sn.pagerank_push(10, 0.85)
            assert max_rel_err(pr, O.pagerank_push(0, 10, 0.85)) <= PR_TOL


def test_push_device_output_and_zero_iterations():
    import torch
    spec = workloads.rmat_single_level(scale=13, seed=5)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            host = sn.pagerank_push(8, 0.85)
            dev = torch.empty(hg.max_nodes, dtype=torch.float64, device="cuda")
            sn.pagerank_push(8, 0.85, out=dev)
            st.sync()
            assert max_rel_err(dev.cpu().numpy(), host) <= PR_TOL
            pr0 = sn.pagerank_push(0, 0.85)
            assert np.all(pr0 == 1.0 / hg.max_nodes)
            with pytest.raises(lb.LgError):
                sn.pagerank_push(5, 1.5)
