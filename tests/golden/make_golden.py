"""Generate the golden fixtures in tests/golden/ by running the REFERENCE.

The reference (goatdb/llama) ships no golden vectors or expected outputs, so
these fixtures come from its own code: oracle/_ref/libllref.so is built from
the reference's headers (oracle/Makefile) and ref_harness.cc builds every
level through the reference's CSR API and runs its benchmark kernels.

Each fixture stores the level inputs (new edges and deletions per level) and
what the reference produced from them: the vertex table and edge-table slots
of every level, the adjacency of every snapshot in iteration order, degrees,
PageRank (pagerank_double) and BFS levels (sssp_unweighted).

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
    levels = [hg.level_input(l)[:4] for l in range(hg.num_levels)]
    return spec.max_nodes, levels


def handmade():
    """Tiny store exercising the corner cases of init_node / iter_descend:
    a vertex whose out-degree drops to zero and comes back, a deletion-only
    vertex (its continuation space is written but never read), a level with
    deletions only, a level with no change at all, vertex 7 isolated."""
    V = 8
    e = lambda pairs: (np.array([p[0] for p in pairs], np.uint32),  # noqa: E731
                       np.array([p[1] for p in pairs], np.uint32))
    none = np.zeros(0, np.uint32)
    l0 = e([(0, 1), (0, 2), (0, 3), (1, 2), (2, 0), (3, 4), (4, 5), (5, 3)])
    l1 = e([(0, 4), (1, 3), (6, 0)])
    d1 = e([(0, 2), (3, 4)])                 # 3 loses its only edge
    l2 = (none, none)
    d2 = e([(1, 2), (0, 1)])                 # deletions only
    l3 = e([(3, 0), (3, 6), (1, 2)])         # 3 comes back; (1,2) re-added
    l4 = (none, none)                        # nothing changes
    return V, [(l0[0], l0[1], none, none), (l1[0], l1[1], d1[0], d1[1]),
               (l2[0], l2[1], d2[0], d2[1]), (l3[0], l3[1], none, none),
               (l4[0], l4[1], none, none)]


CASES = {
    "handmade_5level": handmade,
    "rmat10_1level": lambda: generated(workloads.rmat_single_level(scale=10, seed=1)),
    "rmat10_4level_del": lambda: generated(workloads.rmat_multiversion(
        scale=10, seed=2, levels=4, level0=0.7, delete=0.05)),
    "rmat9_8level_heavydel": lambda: generated(workloads.rmat_multiversion(
        scale=9, seed=3, levels=8, level0=0.5, delete=0.2)),
    "kron9_sym_4level": lambda: generated(workloads.kronecker_symmetric(scale=9, seed=6, levels=4)),
}


def roots_for(V, seed):
    rng = np.random.default_rng(seed)
    return np.unique(np.concatenate([[0], rng.integers(0, V, 3)])).astype(np.int64)


def make(name, fn):
    V, levels = fn()
    R = Reference(V)
    out = {"V": np.int64(V), "num_levels": np.int64(len(levels)),
           "pr_iters": np.int64(PR_ITERS), "damping": np.float64(DAMPING)}
    for l, (s, d, ds, dd) in enumerate(levels):
        R.add_level(s, d, ds, dd)
        out[f"in{l}_src"], out[f"in{l}_dst"] = s, d
        out[f"in{l}_dsrc"], out[f"in{l}_ddst"] = ds, dd
    roots = roots_for(V, 11)
    out["roots"] = roots
    for l in range(len(levels)):
        # level arrays of the full store (later levels' deletion marks included)
        for dr in (0, 1):
            vt, sl = R.level_arrays(l, dr)
            out[f"vt{l}_{dr}"] = vt.view(np.uint8)
            out[f"slots{l}_{dr}"] = sl
        # snapshot l = a reference store holding exactly levels 0..l, queried
        # at its latest level (what `benchmark -l` loads)
        S = Reference(V)
        for (s, d, ds, dd) in levels[:l + 1]:
            S.add_level(s, d, ds, dd)
        for dr in (0, 1):
            off, nb = S.adjacency(-1, dr)
            out[f"adj{l}_{dr}_off"], out[f"adj{l}_{dr}_nbr"] = off, nb
        out[f"outdeg{l}"] = S.degrees(-1)
        out[f"pr{l}"], _ = S.pagerank_pull(-1, PR_ITERS, DAMPING)
        out[f"bfs{l}"] = np.stack([S.bfs(-1, r)[0] for r in roots])
        out[f"bfscount{l}"] = np.array([S.bfs_count(-1, r)[0] for r in roots])
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: V={V} levels={len(levels)} {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    for name, fn in CASES.items():
        make(name, fn)
