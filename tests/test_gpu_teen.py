"""Task avg_teen_cnt on the GPU against the reference's in-adjacency (golden
fixtures) and the oracle: counts exact, average equal."""
import numpy as np
import pytest

from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle
from tests.test_golden_oracle import teen_expected

pytestmark = pytest.mark.gpu


def test_golden_avg_teen_cnt(golden):
    V = int(golden["V"])
    hg = HostGraph(V)
    for lv in golden["levels"]:
        hg.add_level(*lv)
    rng = np.random.default_rng(22)
    age = rng.integers(0, 40, V).astype(np.int32)
    with Store() as st:
        st.ingest(hg)
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                exp = teen_expected(golden[f"adj{l}_1_off"], golden[f"adj{l}_1_nbr"], age, 15)
                for flat in (False, True):
                    if flat:
                        sn.flatten(1)
                    cnt, r = sn.avg_teen_cnt(age, 15)
                    assert np.array_equal(cnt, exp[0]), (l, flat)
                    assert (r.average, r.teen_sum, r.vertices) == exp[1:], (l, flat)


@pytest.mark.parametrize("K", [0, 30, 1000])
def test_avg_teen_cnt_multiversion_vs_oracle(K):
    spec = workloads.rmat_multiversion(scale=15, seed=5, levels=6, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    age = np.random.default_rng(K + 1).integers(0, 80, hg.max_nodes).astype(np.int32)
    with Store() as st:
        st.ingest(hg)
        for l in (0, 5):
            with st.snapshot(l) as sn:
                cnt, r = sn.avg_teen_cnt(age, K)
                avg, ocnt, S, c = O.avg_teen_cnt(l, age, K)
                assert np.array_equal(cnt, ocnt)
                assert (r.average, r.teen_sum, r.vertices) == (avg, S, c)
                if K == 1000:
                    assert r.vertices == 0 and r.average == 0.0


def test_avg_teen_cnt_device_buffers():
    import torch
    spec = workloads.rmat_single_level(scale=14, seed=6)
    hg = HostGraph.from_spec(spec)
    age = np.random.default_rng(7).integers(0, 30, hg.max_nodes).astype(np.int32)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            host_cnt, hr = sn.avg_teen_cnt(age, 12)
            dev_age = torch.from_numpy(age).cuda()
            dev_cnt = torch.empty(hg.max_nodes, dtype=torch.int32, device="cuda")
            _, dr = sn.avg_teen_cnt(dev_age, 12, out=dev_cnt)
            st.sync()
            assert np.array_equal(dev_cnt.cpu().numpy(), host_cnt)
            assert (dr.average, dr.teen_sum, dr.vertices) == \
                (hr.average, hr.teen_sum, hr.vertices)
