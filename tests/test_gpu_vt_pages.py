"""Level ingest through the copy-on-write page table (lg_csr_level.vt_pages).

LLAMA holds every vertex-table level above 0 as ll_mem_array_swcow pages of
512 elements: a level's page is the previous level's page until cow_write
copies it (llama/include/llama/ll_mem_array.h:1019-1032, 1089-1171).  Here the
host builder's levels are cut into such pages, and every page whose contents
did not change is the very buffer of the level below, so consecutive page
tables share pages as the reference's do.  A store fed this way must hold the
same graph as one fed the flat tables: same adjacency, degrees and results at
every snapshot."""
import ctypes as C

import numpy as np
import pytest

from llama_b200 import HostGraph, Store, workloads

pytestmark = pytest.mark.gpu

PAGE = 512
PAGE_BYTES = PAGE * 16


def paged_levels(hg):
    """Level descriptors of hg with vt replaced by COW page tables; returns
    (descs, keep-alive buffers, shared page count)."""
    descs, keep, shared = [], [], 0
    prev = {0: [], 1: []}
    for l in range(hg.num_levels):
        d = hg.level_desc(l)
        for dirn in (0, 1):
            c = d.out if dirn == 0 else d.in_
            n = (c.max_nodes + 1) * 16
            vt = np.ctypeslib.as_array(C.cast(c.vt, C.POINTER(C.c_uint8)), (n,))
            npages = (c.max_nodes + 1 + PAGE - 1) // PAGE
            pages = []
            for p in range(npages):
                chunk = vt[p * PAGE_BYTES:(p + 1) * PAGE_BYTES]
                old = prev[dirn][p] if p < len(prev[dirn]) else None
                if old is not None and np.array_equal(old[:len(chunk)], chunk):
                    pages.append(old)                    # not written: shared
                    shared += 1
                else:
                    buf = np.zeros(PAGE_BYTES, np.uint8)  # cow_write: a new page
                    buf[:len(chunk)] = chunk
                    pages.append(buf)
            prev[dirn] = pages
            table = (C.c_void_p * npages)(*[pg.ctypes.data for pg in pages])
            keep.extend(pages)
            keep.append(table)
            c.vt = None
            c.vt_pages = C.cast(table, C.c_void_p)
        descs.append(d)
    return descs, keep, shared


def block_levels():
    """Level 0 = a seeded R-MAT graph minus 30 % of the edges among vertices
    below 2048; levels 1-3 add those back in thirds and each deletes 2 % of
    the other level-0 edges of that block, so every level changes the vertex
    tables of the first four pages only and the later pages stay shared."""
    g0 = HostGraph.from_spec(workloads.rmat_single_level(scale=14, seed=3))
    src, dst = g0.level_input(0)[:2]
    rng = np.random.default_rng(7)
    block = (src < 2048) & (dst < 2048)
    held = block & (rng.random(len(src)) < 0.3)
    part = rng.integers(1, 4, len(src))
    gone = np.zeros(len(src), bool)
    hg = HostGraph(g0.max_nodes)
    hg.add_level(src[~held], dst[~held])
    for l in (1, 2, 3):
        cand = np.flatnonzero(block & ~held & ~gone)
        d = rng.choice(cand, max(1, len(cand) // 50), replace=False)
        gone[d] = True
        add = held & (part == l)
        hg.add_level(src[add], dst[add], src[np.sort(d)], dst[np.sort(d)])
    return hg


def test_page_table_ingest_equals_flat_ingest():
    hg = block_levels()
    descs, keep, shared = paged_levels(hg)
    assert shared > 0                                   # pages really are shared
    with Store() as flat, Store() as paged:
        flat.ingest(hg)
        for d in descs:
            paged.ingest_level(d)
        assert paged.num_levels == flat.num_levels == hg.num_levels
        for level in range(hg.num_levels):
            with flat.snapshot(level) as a, paged.snapshot(level) as b:
                for direction in (0, 1):
                    oa, na = a.adjacency(direction)
                    ob, nb = b.adjacency(direction)
                    assert np.array_equal(oa, ob) and np.array_equal(na, nb)
                assert np.array_equal(a.out_degrees(), b.out_degrees())
                assert np.array_equal(a.in_degrees(), b.in_degrees())
                assert np.array_equal(a.pagerank_pull(10, 0.85), b.pagerank_pull(10, 0.85))
                root = int(np.flatnonzero(a.out_degrees())[0])
                assert np.array_equal(a.bfs(root)[0], b.bfs(root)[0])
    del keep
