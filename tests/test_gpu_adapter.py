"""The LLAMA-side binding (llama_b200/adapter/lg_llama_adapter.h), compiled
against the reference's own benchmark headers (oracle/_ref/libllref_gpu.so,
built by oracle/Makefile from oracle/adapter_harness.cc), run as LLAMA would
run it: the graph's levels go to a device store through
lg_llama_ingest_level, then the ll_b_pagerank_pull_gpu task is initialized,
run and finalized.  Its ranks and its finalize() value must be those of the
reference's own pagerank_double task on the same graph."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libllref_gpu.so")


def lib():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libllref_gpu.so not built (needs the reference tree)")
    L = C.CDLL(LIB)
    L.llref_create.restype = C.c_void_p
    L.llref_create.argtypes = [C.c_uint64]
    L.llref_destroy.argtypes = [C.c_void_p]
    L.llref_add_level.restype = C.c_int
    L.llref_add_level.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                  C.c_void_p, C.c_void_p, C.c_uint64]
    L.llref_gpu_pagerank.restype = C.c_int
    L.llref_gpu_pagerank.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
    return L


def u32(a):
    return np.ascontiguousarray(a, np.uint32)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("iters", [1, 10])
def test_gpu_task_equals_reference_task(path, iters):
    L = lib()
    g = load_golden(path)
    V = int(g["V"])
    h = L.llref_create(V)
    try:
        for src, dst, ds, dd, _ in g["levels"]:
            s, d = u32(src), u32(dst)
            order = np.lexsort((d, s))
            s, d = np.ascontiguousarray(s[order]), np.ascontiguousarray(d[order])
            ds, dd = u32(ds), u32(dd)
            assert L.llref_add_level(h, s.ctypes.data, d.ctypes.data, len(s), ds.ctypes.data,
                                     dd.ctypes.data, len(ds)) == 0
        rg = np.empty(V, np.float64)
        rc = np.empty(V, np.float64)
        out = np.empty(3, np.float64)
        assert L.llref_gpu_pagerank(h, iters, 0.85, rg.ctypes.data, rc.ctypes.data,
                                    out.ctypes.data) == 0
        assert out[0] == 0.0                                  # run() succeeded
        assert np.max(np.abs(rg - rc) / np.abs(rc)) <= 1e-12
        assert abs(out[1] - out[2]) <= 1e-12 * abs(out[2])    # finalize(): sum of ranks
    finally:
        L.llref_destroy(h)
