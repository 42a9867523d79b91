"""The oracle's at-size helpers against the oracle's own serial functions.

bench.py checks the full-size workloads with functions that work on plain CSR
arrays in parallel (oracle/lgo.cpp: lgo_csr_tc, lgo_csr_ppr) and builds the
reference arm's inputs with the oracle's generator (lgo_gen_create), so that
the reference process never loads the engine.  These tests pin each helper
on small graphs: the generator against the engine's host builder, the CSR
functions against the store-walking oracle (itself pinned to the reference).
"""
import numpy as np
import pytest

from llama_b200 import HostGraph, workloads
from llama_b200.graph import GraphSpec
from oracle.bind import Oracle, csr_ppr, csr_triangles, generate_levels

SPECS = [
    workloads.rmat_multiversion(scale=11, seed=2, levels=8, level0=0.9, delete=0.02,
                                weight_max=255),
    workloads.kronecker_symmetric(scale=10, seed=6, levels=4),
    workloads.rmat_multiversion(scale=12, seed=7, levels=4, level0=0.97, delete=0.01,
                                weight_max=255),
    workloads.rmat_single_level(scale=10, seed=1),
]


def spec_params(spec):
    return {k: getattr(spec, k) for k in GraphSpec.__dataclass_fields__}


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: f"s{s.scale}_k{s.kind}_L{s.num_levels}")
def test_oracle_generator_equals_engine_builder(spec):
    hg = HostGraph.from_spec(spec)
    lv = generate_levels(**spec_params(spec))
    assert len(lv) == hg.num_levels
    for l in range(hg.num_levels):
        a = hg.level_input(l)
        for x, y in zip(a[:4], lv[l][:4]):
            assert np.array_equal(x, y)
        assert (a[4] is None) == (lv[l][4] is None)
        if a[4] is not None:
            assert np.array_equal(a[4], lv[l][4])


def _oracle(spec):
    lv = generate_levels(**spec_params(spec))
    O = Oracle(spec.max_nodes)
    for x in lv:
        O.add_level(*x[:4])
    return O, len(lv)


@pytest.mark.parametrize("spec", SPECS[:3], ids=lambda s: f"s{s.scale}_k{s.kind}")
def test_csr_triangles_equal_oracle_tc(spec):
    O, L = _oracle(spec)
    for level in range(L):
        off, nb, _ = O.adjacency(level, 0)
        assert csr_triangles(O.V, off, nb) == O.tc(level)


def test_csr_triangles_small_cases():
    # a 4-clique plus a pendant edge and a self-loop, arcs in one direction only
    src = np.array([0, 0, 0, 1, 1, 2, 3, 4], np.uint32)
    dst = np.array([1, 2, 3, 2, 3, 3, 4, 4], np.uint32)
    V = 5
    off = np.zeros(V + 1, np.uint64)
    np.add.at(off, src.astype(np.int64) + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    assert csr_triangles(V, off, dst) == 4
    assert csr_triangles(V, np.zeros(V + 1, np.uint64), np.zeros(0, np.uint32)) == 0


@pytest.mark.parametrize("spec", SPECS[:2], ids=lambda s: f"s{s.scale}_k{s.kind}")
def test_csr_ppr_equals_oracle_ppr(spec):
    O, L = _oracle(spec)
    level = L - 1
    off, nb, _ = O.adjacency(level, 1)
    od = O.degrees(level, 0)
    seeds = workloads.pick_roots(od, 5, seed=3)
    want = O.ppr(level, seeds, 7, 0.85)
    got = csr_ppr(O.V, off, nb, od, seeds, 7, 0.85)
    assert np.array_equal(got, want)        # same order of additions: bit for bit


@pytest.mark.parametrize("spec", SPECS[:2], ids=lambda s: f"s{s.scale}_k{s.kind}")
def test_csr_bc_equals_oracle_bc(spec):
    from oracle.bind import csr_bc
    O, L = _oracle(spec)
    level = L - 1
    off, nb, _ = O.adjacency(level, 0)
    src = workloads.pick_roots(O.degrees(level, 0), 6, seed=4)
    want = O.bc(level, src)
    got = csr_bc(O.V, off, nb, src)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_csr_from_edges_keeps_order():
    from oracle.bind import csr_from_edges
    src = np.array([2, 0, 2, 1, 0], np.uint32)
    dst = np.array([5, 6, 7, 8, 9], np.uint32)
    off, nb = csr_from_edges(4, src, dst)
    assert off.tolist() == [0, 2, 3, 5, 5]
    assert nb.tolist() == [6, 9, 8, 5, 7]


@pytest.mark.skipif(not __import__("oracle.bind", fromlist=["ref_available"]).ref_available(),
                    reason="oracle/_ref not built")
def test_reference_weighted_levels_match_the_oracle():
    # the reference harness writes each vertex's new-edge weights by edge id
    # from the vertex's first new edge; its sssp_weighted must see the
    # weights the oracle stores per slot
    from oracle.bind import Reference
    spec = SPECS[2]
    lv = generate_levels(**spec_params(spec))
    R = Reference(spec.max_nodes)
    O = Oracle(spec.max_nodes)
    for x in lv:
        R.add_level(*x)
        O.add_level(*x)
    L = len(lv) - 1
    for r in workloads.pick_roots(O.degrees(L, 0), 4, seed=9):
        want, _ = O.sssp(L, int(r))
        got, _ = R.sssp(-1, int(r))
        assert np.array_equal(got, want)
