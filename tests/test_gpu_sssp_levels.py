"""One-launch delta-stepping (LG_TUNE_SSSP_LEVELS = 1: all rounds, bucket
splits and heavy phases in one cooperative launch) against the per-step host
loop (0), the oracle and the reference's golden distances: distances bit for
bit and the same result fields (both apply the same rules in the same
order), with and without the light/heavy split."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from llama_b200.graph import tune_reset, tune_set
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu


def _fields(r):
    return (r.reached, r.reach_edges, r.max_dist)


def _both(sn, root, delta):
    tune_set(0, "sssp_levels", 0)
    a, ra = sn.sssp(int(root), delta)
    tune_set(0, "sssp_levels", 1)
    b, rb = sn.sssp(int(root), delta)
    return a, ra, b, rb


def test_golden(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    with Store() as st:
        st.ingest(hg)
        try:
            for l in range(len(golden["levels"])):
                with st.snapshot(l) as sn:
                    for split in (0, 1):
                        tune_set(0, "sssp_split", split)
                        for i, r in enumerate(golden["roots"]):
                            for delta in (1, 32, 1 << 20):
                                a, ra, b, rb = _both(sn, r, delta)
                                assert np.array_equal(b, golden[f"sssp{l}"][i]), (l, r, delta)
                                assert np.array_equal(a, b)
                                assert _fields(ra) == _fields(rb), (l, r, delta, split)
        finally:
            tune_reset(0)


@pytest.mark.parametrize("scale,delta", [(12, 32), (15, 32), (15, 7)])
def test_matches_loop_and_oracle(scale, delta):
    spec = workloads.rmat_multiversion(scale=scale, seed=scale + delta, levels=4, level0=0.85,
                                       delete=0.01, weight_max=255)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l))
    with Store() as st:
        st.ingest(hg)
        try:
            with st.snapshot() as sn:
                deg = sn.out_degrees()
                roots = list(workloads.pick_roots(deg, 6, seed=4))
                roots.append(int(np.argmin(deg)))            # a root without out-edges
                for flat in (False, True):
                    if flat:
                        sn.flatten(0)
                    for split in (0, 1):
                        tune_set(0, "sssp_split", split)
                        for k, r in enumerate(roots):
                            a, ra, b, rb = _both(sn, r, delta)
                            assert np.array_equal(a, b), (r, flat, split)
                            assert _fields(ra) == _fields(rb), (r, flat, split)
                            if k % 3 == 0 and delta == 32:
                                ref, reached = O.sssp(hg.num_levels - 1, int(r))
                                assert np.array_equal(b, ref)
                                assert rb.reached == reached
        finally:
            tune_reset(0)


def test_device_output_and_repeats():
    import torch
    spec = workloads.rmat_multiversion(scale=14, seed=2, levels=3, level0=0.9, delete=0.01,
                                       weight_max=255)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            roots = workloads.pick_roots(sn.out_degrees(), 4, seed=6)
            tune_set(0, "sssp_levels", 0)
            want = [sn.sssp(int(r), 32)[0] for r in roots]
            tune_set(0, "sssp_levels", 1)
            out = torch.empty(sn.max_nodes, dtype=torch.int32, device="cuda")
            try:
                for _ in range(2):
                    for r, w in zip(roots, want):
                        assert np.array_equal(sn.sssp(int(r), 32)[0], w)
                        sn.sssp(int(r), 32, out=out)
                        st.sync()
                        assert np.array_equal(out.cpu().numpy(), w)
            finally:
                tune_reset(0)
