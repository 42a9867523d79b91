"""One-launch BFS (LG_TUNE_BFS_LEVELS = 1: every level of lg_bfs in one
cooperative launch, directions chosen on the device) against the per-level
launch loop (0), the oracle and the reference's golden levels: levels bit for
bit, and the same result fields (reached, reach_edges, max_level and the
top-down / bottom-up step counts, since both make the same choices)."""
import numpy as np
import pytest

from llama_b200 import HostGraph, Store, workloads
from llama_b200.graph import tune_reset, tune_set
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu


def _fields(r):
    return (r.reached, r.reach_edges, r.max_level, r.top_down_steps, r.bottom_up_steps)


def _both(sn, root):
    tune_set(0, "bfs_levels", 0)
    a, ra = sn.bfs(int(root))
    tune_set(0, "bfs_levels", 1)
    b, rb = sn.bfs(int(root))
    tune_reset(0)
    return a, ra, b, rb


def test_golden_levels(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    with Store() as st:
        st.ingest(hg)
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                sn.flatten(1)
                for flat_out in (False, True):
                    if flat_out:
                        sn.flatten(0)
                    for i, r in enumerate(golden["roots"]):
                        a, ra, b, rb = _both(sn, r)
                        assert np.array_equal(b, golden[f"bfs{l}"][i]), (l, i, flat_out)
                        assert np.array_equal(a, b)
                        assert _fields(ra) == _fields(rb)
                        assert rb.reached == golden[f"bfscount{l}"][i]


@pytest.mark.parametrize("scale,levels,delete", [(12, 3, 0.05), (15, 6, 0.01)])
def test_matches_loop_and_oracle(scale, levels, delete):
    spec = workloads.rmat_multiversion(scale=scale, seed=scale, levels=levels, level0=0.85,
                                       delete=delete)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    L = hg.num_levels - 1
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            deg = sn.out_degrees()
            roots = list(workloads.pick_roots(deg, 24, seed=5))
            roots.append(int(np.argmin(deg)))             # a root without out-edges
            sn.flatten(1)
            saw_bu = False
            for k, r in enumerate(roots):
                if k == 12:
                    sn.flatten(0)                         # the rest over the flat out-CSR
                a, ra, b, rb = _both(sn, r)
                assert np.array_equal(a, b), r
                assert _fields(ra) == _fields(rb), r
                saw_bu |= rb.bottom_up_steps > 0
                if k % 4 == 0:
                    ref, reached = O.bfs(L, int(r))
                    assert np.array_equal(b, ref)
            assert saw_bu                                 # both directions ran


def test_repeated_calls_and_device_output():
    """Back-to-back calls reuse the control block and the scratch buffers;
    a device output array gets the same levels."""
    import torch
    spec = workloads.rmat_multiversion(scale=14, seed=3, levels=4, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            sn.flatten(1)
            roots = workloads.pick_roots(sn.out_degrees(), 6, seed=8)
            tune_set(0, "bfs_levels", 0)
            want = [sn.bfs(int(r))[0] for r in roots]
            tune_set(0, "bfs_levels", 1)
            out = torch.empty(sn.max_nodes, dtype=torch.int32, device="cuda")
            for _ in range(3):
                for r, w in zip(roots, want):
                    assert np.array_equal(sn.bfs(int(r))[0], w)
                    sn.bfs(int(r), out=out)
                    st.sync()
                    assert np.array_equal(out.cpu().numpy(), w)
            tune_reset(0)


def test_no_in_csr_runs_top_down_only():
    """Top-down only: frontiers of more than 2048 vertices take the scan over
    barrier-separated phases, smaller ones the scan every CTA forms itself."""
    spec = workloads.rmat_single_level(scale=15, seed=4)
    hg = HostGraph.from_spec(spec, reverse_edges=False)
    with Store(reverse_edges=False) as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            big = False
            for r in workloads.pick_roots(sn.out_degrees(), 6, seed=2):
                a, ra, b, rb = _both(sn, r)
                assert np.array_equal(a, b)
                assert _fields(ra) == _fields(rb)
                assert rb.bottom_up_steps == 0
                big |= np.bincount(b[b != 2147483646]).max() > 2048
            assert big
