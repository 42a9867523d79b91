"""Seeded synthetic workloads, named by what they are.

Inputs are the builder's own seeded generators (no dataset is read):
R-MAT with a/b/c/d = 0.57/0.19/0.19/0.05, no noise, self-loops and duplicate
edges removed; edge_factor * 2^scale draws before de-duplication.
"""
import numpy as np

from ._lib import LG_GEN_KRONECKER
from .graph import GraphSpec


def rmat_single_level(scale=16, seed=1):
    """Directed R-MAT, one level (the small CPU-runnable case at scale 16)."""
    return GraphSpec(scale=scale, seed=seed, num_levels=1, level0_fraction=1.0)


def rmat_multiversion(scale=24, seed=2, levels=8, level0=0.90, delete=0.002,
                      weight_max=0):
    """Directed R-MAT split into `levels` snapshots: a seeded 90 % of the edges
    form level 0, the rest is spread evenly over levels 1..levels-1, and every
    level > 0 deletes `delete` of the edges live before it (deletion marks in
    older levels)."""
    return GraphSpec(scale=scale, seed=seed, num_levels=levels, level0_fraction=level0,
                     delete_fraction=delete, split_seed=seed * 1000 + 17,
                     weight_max=weight_max, weight_seed=seed * 1000 + 29)


def kronecker_symmetric(scale=21, seed=6, levels=4):
    """Undirected Graph500-style Kronecker graph (scrambled ids, both arcs of
    every edge), stored as `levels` snapshots of equal share."""
    return GraphSpec(scale=scale, seed=seed, kind=LG_GEN_KRONECKER, symmetrize=True,
                     num_levels=levels, level0_fraction=1.0 / levels,
                     split_seed=seed * 1000 + 17)


def pick_roots(out_degrees, count, seed):
    """`count` distinct roots with out-degree > 0, drawn with a seeded RNG."""
    cand = np.flatnonzero(np.asarray(out_degrees) > 0)
    rng = np.random.default_rng(seed)
    return rng.choice(cand, size=min(count, len(cand)), replace=False).astype(np.int64)
