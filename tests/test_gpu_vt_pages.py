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


def test_page_table_ingest_equals_flat_ingest():
    spec = workloads.rmat_multiversion(scale=14, seed=3, levels=6, level0=0.9, delete=0.003)
    hg = HostGraph.from_spec(spec)
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
