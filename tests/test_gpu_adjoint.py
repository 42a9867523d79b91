"""Differentiable weighted PageRank on the GPU (lg_pagerank_fwd / _bwd):
forward against a dense FP64 solve and the oracle, gradients against the
oracle's adjoint and FP64 central finite differences (h = 1e-6)."""
import numpy as np
import pytest

from llama_b200 import HostGraph, Store, workloads
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu


def setup_graph(scale, seed, levels=3):
    spec = workloads.rmat_multiversion(scale=scale, seed=seed, levels=levels, level0=0.8,
                                       delete=0.02)
    hg = HostGraph.from_spec(spec)
    O = Oracle(hg.max_nodes)
    for l in range(hg.num_levels):
        O.add_level(*hg.level_input(l)[:4])
    return spec, hg, O


def weights_and_teleport(O, level, seed):
    off, nb, _ = O.adjacency(level, 0)
    V = O.V
    rng = np.random.default_rng(seed)
    raw = rng.uniform(0.5, 1.5, len(nb))
    src = np.repeat(np.arange(V), np.diff(off.astype(np.int64)))
    w = raw / np.bincount(src, raw, V)[src]          # row-normalised
    v = rng.exponential(1.0, V)
    v /= v.sum()                                     # Dirichlet(1)
    return w, v, src, nb.astype(np.int64)


def test_forward_matches_dense_solve_and_oracle():
    spec, hg, O = setup_graph(9, 4)
    L = hg.num_levels - 1
    w, v, src, dst = weights_and_teleport(O, L, 1)
    V, d = hg.max_nodes, 0.85
    P = np.zeros((V, V))
    np.add.at(P, (src, dst), w)
    dense = np.linalg.solve(np.eye(V) - d * P.T, (1 - d) * v)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            x, tape, res = sn.pagerank_fwd(w, v, d, tol=1e-12)
            tape.close()
            assert res.residual < 1e-12
            assert np.abs(x - dense).max() < 1e-11
            ox, _ = O.wpr_forward(L, w, v, d)
            assert np.abs(x - ox).sum() < 1e-10


def test_gradients_match_oracle_and_finite_differences():
    spec, hg, O = setup_graph(10, 5)
    L = hg.num_levels - 1
    w, v, src, dst = weights_and_teleport(O, L, 2)
    V, d = hg.max_nodes, 0.85
    rng = np.random.default_rng(3)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            u, _, _ = sn.pagerank_fwd(w, np.full(V, 1.0 / V), d, keep_tape=False)
            T = rng.choice(V, 64, replace=False)
            tgt = 1.2 * u[T]

            def loss(x):
                return float(np.sum((x[T] - tgt) ** 2))

            x, tape, _ = sn.pagerank_fwd(w, v, d)
            g = np.zeros(V)
            g[T] = 2.0 * (x[T] - tgt)
            dw, dv, res = tape.backward(g)
            tape.close()
            ow, ov, _ = O.wpr_backward(L, w, x, g, d)
            assert np.max(np.abs(dw - ow)) <= 1e-9 * np.max(np.abs(ow))
            assert np.max(np.abs(dv - ov)) <= 1e-9 * np.max(np.abs(ov))
            h = 1e-6
            for e in rng.choice(len(w), 16, replace=False):
                wp, wm = w.copy(), w.copy()
                wp[e] += h
                wm[e] -= h
                fd = (loss(sn.pagerank_fwd(wp, v, d, keep_tape=False)[0])
                      - loss(sn.pagerank_fwd(wm, v, d, keep_tape=False)[0])) / (2 * h)
                assert abs(dw[e] - fd) <= 1e-6 * max(abs(fd), 1e-12) + 1e-12, e
            for t in rng.choice(V, 16, replace=False):
                vp, vm = v.copy(), v.copy()
                vp[t] += h
                vm[t] -= h
                fd = (loss(sn.pagerank_fwd(w, vp, d, keep_tape=False)[0])
                      - loss(sn.pagerank_fwd(w, vm, d, keep_tape=False)[0])) / (2 * h)
                assert abs(dv[t] - fd) <= 1e-6 * max(abs(fd), 1e-12) + 1e-12, t


def test_iteration_count_and_cutoff_match_oracle():
    # the solve issues iterations in chunks and stops on the device: it must
    # stop where a loop that checks every iteration stops, and after exactly
    # max_iter iterations when tol is out of reach
    spec, hg, O = setup_graph(11, 6)
    L = hg.num_levels - 1
    w, v, _, _ = weights_and_teleport(O, L, 3)
    with Store() as st:
        st.ingest(hg)
        with st.snapshot() as sn:
            x, _, res = sn.pagerank_fwd(w, v, 0.85, tol=1e-10, keep_tape=False)
            ox, oit = O.wpr_forward(L, w, v, 0.85, tol=1e-10)
            assert abs(res.iterations - oit) <= 1
            assert np.abs(x - ox).sum() < 1e-9
            for m in (1, 2, 3, 16, 17, 33):
                xm, _, rm = sn.pagerank_fwd(w, v, 0.85, tol=1e-300, max_iter=m,
                                            keep_tape=False)
                oxm, oitm = O.wpr_forward(L, w, v, 0.85, tol=1e-300, max_iter=m)
                assert rm.iterations == m == oitm
                assert np.max(np.abs(xm - oxm)) <= 1e-15, m
