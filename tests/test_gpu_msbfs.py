"""Multi-source BFS (lg_bfs_multi): every row equals the single-root BFS and
the oracle / the reference's golden levels, bit for bit."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu


def test_golden_multi(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    with Store() as st:
        st.ingest(hg)
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                roots = np.asarray(golden["roots"], np.int64)
                for flat in (False, True):
                    if flat:
                        sn.flatten(0)
                        sn.flatten(1)
                    lv, res = sn.bfs_multi(roots)
                    for i in range(len(roots)):
                        assert np.array_equal(lv[i], golden[f"bfs{l}"][i]), (l, i, flat)
                        assert res[i].reached == golden[f"bfscount{l}"][i]


@pytest.mark.parametrize("n_roots", [1, 16, 64, 70])
def test_multi_matches_single_and_oracle(n_roots):
    spec = workloads.rmat_multiversion(scale=14, seed=9, levels=5, level0=0.85, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    L = hg.num_levels - 1
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            deg = sn.out_degrees()
            roots = workloads.pick_roots(deg, min(n_roots, 60), seed=n_roots)
            roots = np.resize(roots, n_roots).astype(np.int64)   # repeats past 60
            roots[-1] = int(np.argmin(deg))                      # a root without out-edges
            sn.flatten(1)
            lv, res = sn.bfs_multi(roots)
            for i, r in enumerate(roots):
                one, r1 = sn.bfs(int(r))
                assert np.array_equal(lv[i], one), i
                assert res[i].reached == r1.reached and res[i].reach_edges == r1.reach_edges
                assert res[i].max_level == r1.max_level
            for i in range(0, n_roots, max(1, n_roots // 5)):
                ref, reached = O.bfs(L, int(roots[i]))
                assert np.array_equal(lv[i], ref)


def test_multi_device_output_and_no_in_csr():
    import torch
    spec = workloads.rmat_single_level(scale=13, seed=4)
    hg = HostGraph.from_spec(spec, reverse_edges=False)
    with Store(reverse_edges=False) as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            roots = workloads.pick_roots(sn.out_degrees(), 8, seed=1)
            out = torch.empty((8, sn.max_nodes), dtype=torch.int32, device="cuda")
            sn.bfs_multi(roots, out=out)
            st.sync()
            host, _ = sn.bfs_multi(roots)
            assert np.array_equal(out.cpu().numpy(), host)
            for i, r in enumerate(roots):
                assert np.array_equal(host[i], sn.bfs(int(r))[0])
            with pytest.raises(lb.LgError):
                sn.bfs_multi([sn.max_nodes])
