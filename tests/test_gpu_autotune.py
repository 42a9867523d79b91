"""Launch parameters change speed, never results: every candidate value of
every tunable gives the same output (bit for bit where the summation order
does not depend on it), and lg_autotune measures them on a snapshot and keeps
the fastest."""
import numpy as np
import pytest

from llama_b200 import HostGraph, Store, workloads
from llama_b200.graph import ppr, tune_get, tune_reset, tune_set

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def store():
    spec = workloads.rmat_multiversion(scale=13, seed=11, levels=3, level0=0.9, delete=0.01,
                                       weight_max=255)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        yield st
    tune_reset(0)


def test_every_value_gives_the_same_results(store):
    tune_reset(0)
    with store.snapshot() as sn:
        deg = sn.out_degrees()
        roots = workloads.pick_roots(deg, 64, seed=2)
        seeds = workloads.pick_roots(deg, 128, seed=3)
        pr0 = sn.pagerank_pull(7, 0.85)
        x0 = ppr([sn], seeds, iterations=5)
        lv0, _ = sn.bfs_multi(roots)
        d0, _ = sn.sssp(int(roots[0]), 32)
        for c in (4, 5, 6, 8):
            tune_set(0, "pr_ctas_per_sm", c)
            assert np.array_equal(sn.pagerank_pull(7, 0.85), pr0)
        tune_reset(0)
        tune_set(0, "pr_tile_occ", 8)
        assert np.array_equal(sn.pagerank_pull(7, 0.85), pr0)
        tune_reset(0)
        for kt in (32, 64, 128):
            tune_set(0, "ppr_ktile", kt)
            assert np.array_equal(ppr([sn], seeds, iterations=5), x0)
        tune_reset(0)
        for r in (256, 1024, 4096):
            tune_set(0, "ppr_range", r)
            x = ppr([sn], seeds, iterations=5)
            nz = x0 != 0
            assert np.array_equal(x == 0, ~nz)
            assert np.max(np.abs(x[nz] - x0[nz]) / x0[nz]) <= 1e-12
        tune_reset(0)
        sn.flatten(1)                     # the threshold is read by the flat bottom-up kernels
        for h in (32, 128, 4096):
            tune_set(0, "ms_heavy", h)
            assert np.array_equal(sn.bfs_multi(roots)[0], lv0)
        sn.unflatten()
        tune_reset(0)
        for r in (256, 512, 4096):
            tune_set(0, "sssp_range", r)
            assert np.array_equal(sn.sssp(int(roots[0]), 32)[0], d0)
        tune_reset(0)
        tune_set(0, "sssp_split", 0)
        for r in roots[:4]:
            a = sn.sssp(int(r), 32)[0]
            tune_set(0, "sssp_split", 1)
            assert np.array_equal(sn.sssp(int(r), 32)[0], a)
            assert np.array_equal(sn.sssp(int(r), 7)[0], a)        # another delta
            tune_set(0, "sssp_split", 0)
        tune_reset(0)


def test_autotune_keeps_the_fastest_measured_value(store):
    tune_reset(0)
    with store.snapshot() as sn:
        res = sn.autotune()
        # the flat in-CSR made for the probes is released again
        assert not sn.is_flat(1)
    assert set(res) == {"pr_ctas_per_sm", "ppr_ktile", "ppr_range", "sssp_range", "ms_heavy",
                        "pr_tile_occ", "sssp_split", "bfs_levels", "sssp_levels"}
    for name, r in res.items():
        assert r["chosen"] in r["ms"]
        assert all(ms > 0 for ms in r["ms"].values())
        assert r["ms"][r["chosen"]] == min(r["ms"].values())
        assert tune_get(0, name) == r["chosen"]
    tune_reset(0)


def test_autotune_leaves_a_flat_snapshot_flat(store):
    """A snapshot that was flat before the probes stays flat after them."""
    tune_reset(0)
    with store.snapshot() as sn:
        sn.flatten(1)
        res = sn.autotune(["ms_heavy"])
        assert sn.is_flat(1)
    assert set(res) == {"ms_heavy"}
    assert res["ms_heavy"]["ms"][res["ms_heavy"]["chosen"]] == min(res["ms_heavy"]["ms"].values())
    tune_reset(0)
