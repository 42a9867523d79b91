"""GPU parity: the CUDA engine through the C ABI against the reference's
golden outputs and the CPU oracle.

Bars: adjacency, degrees and BFS levels bit-exact; FP64 PageRank within 1e-12
max relative error (only the summation order differs from the reference).
"""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle
from tests._util import max_rel_err

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12


def device_store(levels, V):
    hg = HostGraph(V)
    for lv in levels:
        hg.add_level(*lv)
    st = Store()
    st.ingest(hg)
    return hg, st


def test_golden_snapshots(golden):
    V = int(golden["V"])
    hg, st = device_store(golden["levels"], V)
    with st:
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                for dr in (0, 1):
                    off, nb = sn.adjacency(dr)
                    assert np.array_equal(off, golden[f"adj{l}_{dr}_off"]), (l, dr)
                    assert np.array_equal(nb, golden[f"adj{l}_{dr}_nbr"]), (l, dr)
                assert np.array_equal(sn.out_degrees(), golden[f"outdeg{l}"])
                pr = sn.pagerank_pull(int(golden["pr_iters"]), float(golden["damping"]))
                assert max_rel_err(pr, golden[f"pr{l}"]) <= PR_TOL, l
                for i, r in enumerate(golden["roots"]):
                    lv, res = sn.bfs(int(r))
                    assert np.array_equal(lv, golden[f"bfs{l}"][i]), (l, r)
                    assert res.reached == golden[f"bfscount{l}"][i]


def _oracle_for(hg):
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    return O


def test_rmat16_single_level_pagerank_bfs():
    """R-MAT scale 16, one level: PageRank FP64 10 iterations, BFS from 0."""
    spec = workloads.rmat_single_level(scale=16, seed=1)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            st1 = sn.stats(1)
            assert st1["ranges"] > 1 and np.max(sn.in_degrees()) > 2048  # straddling vertices
            pr = sn.pagerank_pull(10, 0.85)
            assert max_rel_err(pr, O.pagerank_pull(0, 10, 0.85)) <= PR_TOL
            lv, res = sn.bfs(0)
            ref, reached = O.bfs(0, 0)
            assert np.array_equal(lv, ref)
            assert res.reached == reached


def test_multiversion_with_deletions_every_snapshot():
    spec = workloads.rmat_multiversion(scale=15, seed=2, levels=8, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        for l in (0, 3, 7):
            with st.snapshot(l) as sn:
                off, nb = sn.adjacency(0)
                o_off, o_nb, _ = O.adjacency(l, 0)
                assert np.array_equal(off, o_off) and np.array_equal(nb, o_nb)
                off, nb = sn.adjacency(1)
                o_off, o_nb, _ = O.adjacency(l, 1)
                assert np.array_equal(off, o_off) and np.array_equal(nb, o_nb)
                assert np.array_equal(sn.in_degrees(), O.degrees(l, 1))
                pr = sn.pagerank_pull(20, 0.85)
                assert max_rel_err(pr, O.pagerank_pull(l, 20, 0.85)) <= PR_TOL
                deg = sn.out_degrees()
                for r in workloads.pick_roots(deg, 4, seed=3):
                    lv, res = sn.bfs(int(r))
                    ref, reached = O.bfs(l, int(r))
                    assert np.array_equal(lv, ref), (l, r)
                    assert res.reached == reached


def test_device_outputs_and_reuse():
    """Outputs written straight into torch CUDA tensors; repeated calls agree."""
    import torch
    spec = workloads.rmat_multiversion(scale=14, seed=4, levels=3, level0=0.8, delete=0.02)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            host = sn.pagerank_pull(7)
            dev = torch.empty(sn.max_nodes, dtype=torch.float64, device="cuda")
            sn.pagerank_pull(7, out=dev)
            st.sync()
            assert np.array_equal(dev.cpu().numpy(), host)   # deterministic
            lv_dev = torch.empty(sn.max_nodes, dtype=torch.int32, device="cuda")
            _, r1 = sn.bfs(5, out=lv_dev)
            st.sync()
            lv, r2 = sn.bfs(5)
            assert np.array_equal(lv_dev.cpu().numpy(), lv)
            assert r1.reached == r2.reached


def test_incremental_ingest_and_drop_level():
    spec = workloads.rmat_multiversion(scale=13, seed=5, levels=4, level0=0.7, delete=0.05)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        for l in range(4):
            st.ingest_level(hg.level_desc(l))
            with st.snapshot() as sn:
                assert sn.level == l
                assert max_rel_err(sn.pagerank_pull(5), O.pagerank_pull(l, 5)) <= PR_TOL
        st.drop_level()
        st.drop_level()
        assert st.num_levels == 2
        with st.snapshot() as sn:
            off, nb = sn.adjacency(0)
            o_off, o_nb, _ = O.adjacency(1, 0)
            assert np.array_equal(nb, o_nb)
        st.ingest_level(hg.level_desc(2))
        with st.snapshot() as sn:
            assert max_rel_err(sn.pagerank_pull(5), O.pagerank_pull(2, 5)) <= PR_TOL


def test_errors_are_reported_not_faulted():
    spec = workloads.rmat_single_level(scale=10, seed=1)
    hg = HostGraph.from_spec(spec)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(lb.LgError):
                sn.bfs(1 << 10)
            with pytest.raises(lb.LgError):
                sn.pagerank_pull(3, damping=1.5)
            with pytest.raises(lb.LgError):
                st.drop_level()                   # snapshot still open
        with pytest.raises(lb.LgError):
            st.snapshot(3)
    # a level whose vertex table points past its edge table is rejected
    d = hg.level_desc(0)
    d.out.n_slots = 1
    with Store() as st2:
        with pytest.raises(lb.LgError):
            st2.ingest_level(d)
        assert st2.num_levels == 0
        st2.ingest(hg)                            # the store stays usable
        assert st2.num_levels == 1


def test_golden_sssp(golden):
    V = int(golden["V"])
    hg, st = device_store(golden["levels"], V)
    with st:
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                for flat in (False, True):
                    if flat:
                        sn.flatten(0)           # rounds over the flat out-CSR
                    for i, r in enumerate(golden["roots"]):
                        for delta in (1, 32, 1 << 20):
                            d, res = sn.sssp(int(r), delta)
                            assert np.array_equal(d, golden[f"sssp{l}"][i]), (l, r, delta, flat)
                        assert res.reached == int(np.sum(d < lb._lib.LG_UNREACHED))


def test_sssp_multiversion_weights_vs_oracle():
    spec = workloads.rmat_multiversion(scale=15, seed=7, levels=4, level0=0.85, delete=0.01,
                                       weight_max=255)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l))
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            roots = workloads.pick_roots(sn.out_degrees(), 3, seed=8)
            for flat in (False, True):
                if flat:
                    sn.flatten(0)
                for r in roots:
                    d, res = sn.sssp(int(r), 32)
                    ref, reached = O.sssp(3, int(r))
                    assert np.array_equal(d, ref), (r, flat)
                    assert res.reached == reached


def test_sssp_needs_weights():
    hg = HostGraph.from_spec(workloads.rmat_single_level(scale=8, seed=1))
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            with pytest.raises(lb.LgError):
                sn.sssp(0)


def test_golden_triangles(golden):
    V = int(golden["V"])
    hg, st = device_store(golden["levels"], V)
    with st:
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                assert sn.triangle_count().triangles == golden[f"tc{l}"], l


def test_triangles_multiversion_vs_oracle():
    spec = workloads.rmat_multiversion(scale=14, seed=2, levels=8, level0=0.9, delete=0.01)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        for l in (0, 7):
            with st.snapshot(l) as sn:
                r = sn.triangle_count()
                assert r.triangles == O.tc(l)
                assert r.arcs == sn.num_edges


def test_golden_scc(golden):
    V = int(golden["V"])
    hg, st = device_store(golden["levels"], V)
    with st:
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                lab, res = sn.scc()
                assert np.array_equal(lab, golden[f"scc{l}"]), l
                assert res.components == len(np.unique(lab))


def test_scc_multiversion_vs_oracle():
    spec = workloads.rmat_multiversion(scale=15, seed=9, levels=4, level0=0.8, delete=0.02)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        for l in (1, 3):
            with st.snapshot(l) as sn:
                lab, _ = sn.scc()
                assert np.array_equal(lab, O.scc(l))


BC_TOL = 1e-9


def _bc_close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= BC_TOL * np.maximum(np.abs(b), 1.0))


def test_golden_bc_plain_and_batched(golden):
    """FP64 BC vs the FP64 oracle (1e-9) and the FP32 reference (1e-5)."""
    V = int(golden["V"])
    hg, st = device_store(golden["levels"], V)
    O = Oracle(V)
    O.add_levels(golden["levels"])
    src = golden["bc_sources"]
    with st:
        for l in range(len(golden["levels"])):
            with st.snapshot(l) as sn:
                ref = O.bc(l, src)
                plain = sn.bc(src, batched=False)
                batched = sn.bc(src, batched=True)
                assert _bc_close(plain, ref), l
                assert _bc_close(batched, ref), l
                f32 = golden[f"bc{l}"].astype(np.float64)
                assert np.all(np.abs(batched - f32) <= 1e-5 * np.maximum(np.abs(batched), 1.0))


def test_bc_batched_many_sources_vs_oracle():
    """More than one 64-source batch, repeated sources, a symmetric graph."""
    spec = workloads.kronecker_symmetric(scale=11, seed=6, levels=4)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            src = workloads.pick_roots(sn.out_degrees(), 100, seed=7)
            src = np.concatenate([src, src[:5]])
            ref = O.bc(3, src)
            assert _bc_close(sn.bc(src, batched=True), ref)
            assert _bc_close(sn.bc(src[:20], batched=False), O.bc(3, src[:20]))


def test_ppr_block_all_snapshots_vs_oracle():
    from llama_b200.graph import ppr
    spec = workloads.kronecker_symmetric(scale=11, seed=6, levels=4)
    hg = HostGraph.from_spec(spec)
    O = _oracle_for(hg)
    with Store() as st:
        st.ingest(hg)
        snaps = [st.snapshot(l) for l in range(4)]
        try:
            seeds = workloads.pick_roots(snaps[-1].out_degrees(), 64, seed=11)
            seeds[3] = seeds[7]                       # a repeated seed
            res = ppr(snaps, seeds, iterations=6)
            for l in range(4):
                ref = O.ppr(l, seeds, 6)
                den = np.maximum(np.abs(ref), 1e-300)
                assert np.max(np.abs(res[l] - ref) / den) <= 1e-12, l
            # K = 32 path and iteration count 0
            r0 = ppr(snaps[:1], seeds[:32], iterations=0)
            assert np.array_equal(r0[0], O.ppr(0, seeds[:32], 0))
        finally:
            for s in snaps:
                s.close()


def _write_level_files(golden, tmp_path):
    files = []
    for l, (s, d, ds, dd, w) in enumerate(golden["levels"]):
        p = tmp_path / f"level{l}.net"
        with open(p, "w") as f:
            f.write("# level %d\n" % l)
            for a, b, c in zip(s, d, w):
                f.write(f"{a}\t{b}\t{c}\n")
            for a, b in zip(ds, dd):
                f.write(f"- {a}\t{b}\n")
        files.append(str(p))
    return files


@pytest.mark.parametrize("task", ["pagerank_double", "pagerank_double_push", "bfs_count",
                                  "sssp_weighted", "tc_u"])
def test_cli_return_value_matches_reference(golden, tmp_path, task):
    """`lg_benchmark -r TASK FILE...` prints the reference task's return value."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(lb.LIB_PATH), "lg_benchmark")
    files = _write_level_files(golden, tmp_path)
    L = len(files) - 1
    V = int(golden["V"])
    root = int(golden["roots"][0])
    # -N gives the store the fixture's max_nodes (trailing isolated vertices
    # included), the N of the reference's PageRank
    out = subprocess.run([exe, "-r", task, "-R", str(root), "-n", str(int(golden["pr_iters"])),
                          "-N", str(V)] + files,
                         capture_output=True, text=True, check=True).stdout
    ret = float(out.strip().splitlines()[-1].split(":")[1])
    if task in ("pagerank_double", "pagerank_double_push"):
        key = "pr" if task == "pagerank_double" else "prpush"
        # printed like the reference's "Return value: %lf": 6 decimals
        assert abs(ret - float(np.sum(golden[f"{key}{L}"]))) <= 5e-7 + 1e-12
    elif task == "bfs_count":
        assert ret == golden[f"bfscount{L}"][0]
    elif task == "sssp_weighted":
        assert ret == np.sum(golden[f"sssp{L}"][0] < lb._lib.LG_UNREACHED)
    else:
        assert ret == golden[f"tc{L}"]
