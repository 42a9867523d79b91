"""Generate the golden fixtures in tests/golden/ by running the REFERENCE.

The reference (goatdb/llama) ships no golden vectors or expected outputs, so
these fixtures come from its own code: oracle/_ref/libllref.so is built from
the reference's headers (oracle/Makefile) and ref_harness.cc builds every
level through the reference's CSR API and runs its benchmark kernels.

Each fixture stores the level inputs (new edges with uint32 weights, and
deletions, per level) and what the reference produced from them: the vertex
table and edge-table slots of every level; for every snapshot, its adjacency
in iteration order, degrees, PageRank (pagerank_double and
pagerank_double_push), BFS levels
(sssp_unweighted), weighted SSSP distances (sssp_weighted), Brandes BC from
fixed sources (bc_random's kernel, FP32, one thread: with more threads the
reference's down-edge marking races, ll_bfs_template.h:619-640), and triangle
counts (tc_u on the snapshot flattened to one symmetric level).  SCC labels
come from scipy's strongly-connected-components on the reference adjacency
(the reference's tarjan_scc does not compute SCCs), canonicalised to the
smallest vertex id of each component.

Run from the repo root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from llama_b200 import HostGraph, workloads  # noqa: E402  (input generator only)
from oracle.bind import Reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PR_ITERS = 10
DAMPING = 0.85


def generated(spec):
    hg = HostGraph.from_spec(spec)
    return spec.max_nodes, [hg.level_input(l) for l in range(hg.num_levels)]


def handmade():
    """Tiny store exercising the corner cases of init_node / iter_descend:
    a vertex whose out-degree drops to zero and comes back, a deletion-only
    vertex (its continuation space is written but never read), a level with
    deletions only, a level with no change at all, vertex 7 isolated."""
    V = 8

    def e(pairs):
        s = np.array([p[0] for p in pairs], np.uint32)
        d = np.array([p[1] for p in pairs], np.uint32)
        return s, d, (s * 7 + d * 3) % 11 + 1
    none = np.zeros(0, np.uint32)
    l0 = e([(0, 1), (0, 2), (0, 3), (1, 2), (2, 0), (3, 4), (4, 5), (5, 3)])
    l1 = e([(0, 4), (1, 3), (6, 0)])
    d1 = e([(0, 2), (3, 4)])                 # 3 loses its only edge
    d2 = e([(1, 2), (0, 1)])                 # deletions only
    l3 = e([(3, 0), (3, 6), (1, 2)])         # 3 comes back; (1,2) re-added
    return V, [(l0[0], l0[1], none, none, l0[2]), (l1[0], l1[1], d1[0], d1[1], l1[2]),
               (none, none, d2[0], d2[1], none), (l3[0], l3[1], none, none, l3[2]),
               (none, none, none, none, none)]


CASES = {
    "handmade_5level": handmade,
    "rmat10_1level": lambda: generated(workloads.rmat_multiversion(
        scale=10, seed=1, levels=1, level0=1.0, delete=0.0, weight_max=255)),
    "rmat10_4level_del": lambda: generated(workloads.rmat_multiversion(
        scale=10, seed=2, levels=4, level0=0.7, delete=0.05, weight_max=255)),
    "rmat9_8level_heavydel": lambda: generated(workloads.rmat_multiversion(
        scale=9, seed=3, levels=8, level0=0.5, delete=0.2, weight_max=255)),
    "kron9_sym_4level": lambda: generated(workloads.kronecker_symmetric(scale=9, seed=6, levels=4)),
}


def roots_for(V, seed):
    rng = np.random.default_rng(seed)
    return np.unique(np.concatenate([[0], rng.integers(0, V, 3)])).astype(np.int64)


def flatten_symmetric(V, off, nb):
    """One-level symmetric edge list of a snapshot, no self-loops, sorted."""
    src = np.repeat(np.arange(V, dtype=np.uint64), np.diff(off.astype(np.int64)))
    a = np.concatenate([src, nb.astype(np.uint64)])
    b = np.concatenate([nb.astype(np.uint64), src])
    k = np.unique((a << np.uint64(32)) | b)
    k = k[(k >> np.uint64(32)) != (k & np.uint64(0xffffffff))]
    return (k >> np.uint64(32)).astype(np.uint32), (k & np.uint64(0xffffffff)).astype(np.uint32)


def scc_min_labels(V, off, nb):
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg
    A = sp.csr_matrix((np.ones(len(nb)), nb.astype(np.int64), off.astype(np.int64)),
                      shape=(V, V))
    n, lab = cg.connected_components(A, directed=True, connection="strong")
    mins = np.full(n, np.iinfo(np.int64).max)
    np.minimum.at(mins, lab, np.arange(V))
    return mins[lab]


def make(name, fn):
    V, levels = fn()
    Reference.set_threads(1)
    R = Reference(V)
    out = {"V": np.int64(V), "num_levels": np.int64(len(levels)),
           "pr_iters": np.int64(PR_ITERS), "damping": np.float64(DAMPING)}
    for l, (s, d, ds, dd, w) in enumerate(levels):
        w = np.zeros(len(s), np.uint32) if w is None else w
        R.add_level(s, d, ds, dd, w)
        out[f"in{l}_src"], out[f"in{l}_dst"] = s, d
        out[f"in{l}_dsrc"], out[f"in{l}_ddst"] = ds, dd
        out[f"in{l}_w"] = w
    roots = roots_for(V, 11)
    out["roots"] = roots
    bc_src = roots_for(V, 12)
    out["bc_sources"] = bc_src
    for l in range(len(levels)):
        # level arrays of the full store (later levels' deletion marks included)
        for dr in (0, 1):
            vt, sl = R.level_arrays(l, dr)
            out[f"vt{l}_{dr}"] = vt.view(np.uint8)
            out[f"slots{l}_{dr}"] = sl
        # snapshot l = a reference store holding exactly levels 0..l, queried
        # at its latest level (what `benchmark -l` loads)
        S = Reference(V)
        for (s, d, ds, dd, w) in levels[:l + 1]:
            S.add_level(s, d, ds, dd, np.zeros(len(s), np.uint32) if w is None else w)
        for dr in (0, 1):
            off, nb = S.adjacency(-1, dr)
            out[f"adj{l}_{dr}_off"], out[f"adj{l}_{dr}_nbr"] = off, nb
        out[f"outdeg{l}"] = S.degrees(-1)
        out[f"pr{l}"], _ = S.pagerank_pull(-1, PR_ITERS, DAMPING)
        # one thread: the reference's atomic adds then run in vertex order
        out[f"prpush{l}"], _ = S.pagerank_push(-1, PR_ITERS, DAMPING)
        out[f"bfs{l}"] = np.stack([S.bfs(-1, r)[0] for r in roots])
        out[f"bfscount{l}"] = np.array([S.bfs_count(-1, r)[0] for r in roots])
        out[f"sssp{l}"] = np.stack([S.sssp(-1, r)[0] for r in roots])
        out[f"bc{l}"], _ = S.bc(-1, bc_src)
        off, nb = out[f"adj{l}_0_off"], out[f"adj{l}_0_nbr"]
        T = Reference(V)
        T.add_level(*flatten_symmetric(V, off, nb))
        out[f"tc{l}"] = np.int64(T.tc_u()[0])
        out[f"scc{l}"] = scc_min_labels(V, off, nb)
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: V={V} levels={len(levels)} {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    for name, fn in CASES.items():
        make(name, fn)
