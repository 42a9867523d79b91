"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

``Oracle`` wraps oracle/liblgo.so, the plain restatement of the reference's
multiversioned CSR and kernels (oracle/lgo.cpp).  ``Reference`` wraps
oracle/_ref/libllref.so, the reference's own headers compiled from source with
oracle/ref_harness.cc.  Only tests/, the smoke check and bench.py's CPU
baseline use this module; the llama_b200 package never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LGO_PATH = os.path.join(HERE, "liblgo.so")
REF_PATH = os.path.join(HERE, "_ref", "libllref.so")

_P, _U64, _I64, _INT, _D = C.c_void_p, C.c_uint64, C.c_int64, C.c_int, C.c_double


def _p(a):
    return None if a is None else a.ctypes.data


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


_lgo = None
_ref = None


def lgo():
    global _lgo
    if _lgo is None:
        L = C.CDLL(LGO_PATH)
        for name, res, args in [
            ("lgo_create", _P, [_U64]),
            ("lgo_destroy", None, [_P]),
            ("lgo_num_levels", _INT, [_P]),
            ("lgo_add_level", _INT, [_P, _P, _P, _U64, _P, _P, _U64, _P]),
            ("lgo_level_arrays", _INT, [_P, _INT, _INT, C.POINTER(_P), C.POINTER(_U64),
                                        C.POINTER(_P), C.POINTER(_U64)]),
            ("lgo_adjacency", _U64, [_P, _INT, _INT, _P, _P, _P]),
            ("lgo_degrees", None, [_P, _INT, _INT, _P]),
            ("lgo_pagerank_pull", None, [_P, _INT, _INT, _D, _P]),
            ("lgo_pagerank_push", None, [_P, _INT, _INT, _D, _P]),
            ("lgo_bfs", _U64, [_P, _INT, _I64, _P]),
            ("lgo_bc", None, [_P, _INT, _P, _INT, _P]),
            ("lgo_sssp", _U64, [_P, _INT, _I64, _P]),
            ("lgo_tc", _I64, [_P, _INT]),
            ("lgo_set_min_level", None, [_P, _INT]),
            ("lgo_avg_teen_cnt", _D, [_P, _INT, _P, _INT, _P, C.POINTER(_I64),
                                      C.POINTER(_I64)]),
            ("lgo_scc", None, [_P, _INT, _P]),
            ("lgo_ppr", None, [_P, _INT, _P, _INT, _INT, _D, _P]),
            ("lgo_wpr_forward", _INT, [_P, _INT, _P, _P, _D, _D, _INT, _P]),
            ("lgo_wpr_backward", _INT, [_P, _INT, _P, _P, _P, _D, _D, _INT, _P, _P]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lgo = L
    return _lgo


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_PATH)
        for name, res, args in [
            ("llref_create", _P, [_U64]),
            ("llref_destroy", None, [_P]),
            ("llref_num_levels", _INT, [_P]),
            ("llref_add_level", _INT, [_P, _P, _P, _U64, _P, _P, _U64]),
            ("llref_level_arrays", _I64, [_P, _INT, _INT, _P, _P]),
            ("llref_adjacency", _U64, [_P, _INT, _INT, _P, _P]),
            ("llref_degrees", None, [_P, _INT, _P]),
            ("llref_set_threads", None, [_INT]),
            ("llref_max_threads", _INT, []),
            ("llref_pagerank", _D, [_P, _INT, _INT, _D, _P]),
            ("llref_pagerank_push", _D, [_P, _INT, _INT, _D, _P]),
            ("llref_bfs_levels", _D, [_P, _INT, _I64, _P]),
            ("llref_bfs_count", _D, [_P, _INT, _I64, C.POINTER(_D)]),
            ("llref_add_level_weighted", _INT, [_P, _P, _P, _U64, _P, _P, _U64, _P]),
            ("llref_sssp", _D, [_P, _INT, _I64, _P]),
            ("llref_bc", _D, [_P, _INT, _P, _INT, _P]),
            ("llref_tc_u", _I64, [_P, C.POINTER(_D)]),
            ("llref_tarjan_scc", _D, [_P, _INT]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ref = L
    return _ref


VT_DTYPE = np.dtype([("adj_list_start", "<i8"), ("level_length", "<u4"), ("degree", "<u4")])


class _Base:
    V = 0

    def add_levels(self, levels):
        """levels: iterable of (src, dst, del_src, del_dst[, weights])."""
        for lv in levels:
            self.add_level(*lv)


class Oracle(_Base):
    """Plain restatement of the reference (oracle/lgo.cpp)."""

    def __init__(self, V):
        self.V = int(V)
        self.h = lgo().lgo_create(self.V)

    def __del__(self):
        if getattr(self, "h", None):
            lgo().lgo_destroy(self.h)
            self.h = None

    @property
    def num_levels(self):
        return lgo().lgo_num_levels(self.h)

    def add_level(self, src, dst, del_src=(), del_dst=(), weights=None):
        s, d, ds, dd = _u32(src), _u32(dst), _u32(del_src), _u32(del_dst)
        w = None if weights is None else _u32(weights)
        r = lgo().lgo_add_level(self.h, _p(s), _p(d), len(s), _p(ds), _p(dd), len(ds), _p(w))
        if r != 0:
            raise ValueError("oracle rejected the level")

    def level_arrays(self, level, direction=0):
        vt, nvt, et, net = _P(), _U64(), _P(), _U64()
        if lgo().lgo_level_arrays(self.h, direction, level, C.byref(vt), C.byref(nvt),
                                  C.byref(et), C.byref(net)):
            raise ValueError("no such level")
        v = np.ctypeslib.as_array(C.cast(vt, C.POINTER(C.c_uint8)), (nvt.value * 16,))
        e = (np.ctypeslib.as_array(C.cast(et, C.POINTER(C.c_uint64)), (net.value,))
             if net.value else np.zeros(0, np.uint64))
        return v.copy().view(VT_DTYPE), e.copy()

    def adjacency(self, level, direction=0):
        off = np.empty(self.V + 1, np.uint64)
        n = lgo().lgo_adjacency(self.h, direction, level, _p(off), None, None)
        nb = np.empty(max(n, 1), np.uint32)
        ids = np.empty(max(n, 1), np.int64)
        lgo().lgo_adjacency(self.h, direction, level, _p(off), _p(nb), _p(ids))
        return off, nb[:n], ids[:n]

    def degrees(self, level, direction=0):
        d = np.empty(self.V, np.uint32)
        lgo().lgo_degrees(self.h, direction, level, _p(d))
        return d

    def pagerank_pull(self, level, iterations, damping=0.85):
        out = np.empty(self.V, np.float64)
        lgo().lgo_pagerank_pull(self.h, level, iterations, damping, _p(out))
        return out

    def pagerank_push(self, level, iterations, damping=0.85):
        out = np.empty(self.V, np.float64)
        lgo().lgo_pagerank_push(self.h, level, iterations, damping, _p(out))
        return out

    def bfs(self, level, root):
        out = np.empty(self.V, np.int32)
        reached = lgo().lgo_bfs(self.h, level, int(root), _p(out))
        return out, reached

    def bc(self, level, sources):
        src = np.ascontiguousarray(sources, np.int64)
        out = np.empty(self.V, np.float64)
        lgo().lgo_bc(self.h, level, _p(src), len(src), _p(out))
        return out

    def sssp(self, level, root):
        out = np.empty(self.V, np.uint32)
        reached = lgo().lgo_sssp(self.h, level, int(root), _p(out))
        return out, reached

    def tc(self, level):
        return lgo().lgo_tc(self.h, level)

    def set_min_level(self, m):
        """Sliding window: iteration ends at fragments of levels below m."""
        lgo().lgo_set_min_level(self.h, int(m))

    def avg_teen_cnt(self, level, age, K=0):
        """(average, teen_cnt, sum, count) of task avg_teen_cnt."""
        a = np.ascontiguousarray(age, dtype=np.int32)
        out = np.zeros(self.V, np.int32)
        S, c = _I64(), _I64()
        avg = lgo().lgo_avg_teen_cnt(self.h, level, _p(a), int(K), _p(out), C.byref(S),
                                     C.byref(c))
        return avg, out, S.value, c.value

    def scc(self, level):
        out = np.empty(self.V, np.int64)
        lgo().lgo_scc(self.h, level, _p(out))
        return out

    def wpr_forward(self, level, weights, teleport, damping=0.85, tol=1e-12, max_iter=10000):
        w = np.ascontiguousarray(weights, np.float64)
        v = np.ascontiguousarray(teleport, np.float64)
        x = np.empty(self.V, np.float64)
        it = lgo().lgo_wpr_forward(self.h, level, _p(w), _p(v), damping, tol, max_iter, _p(x))
        return x, it

    def wpr_backward(self, level, weights, x, dldx, damping=0.85, tol=1e-12, max_iter=10000):
        w = np.ascontiguousarray(weights, np.float64)
        xx = np.ascontiguousarray(x, np.float64)
        g = np.ascontiguousarray(dldx, np.float64)
        dw = np.empty(len(w), np.float64)
        dv = np.empty(self.V, np.float64)
        it = lgo().lgo_wpr_backward(self.h, level, _p(w), _p(xx), _p(g), damping, tol,
                                    max_iter, _p(dw), _p(dv))
        return dw, dv, it

    def ppr(self, level, seeds, iterations, damping=0.85):
        s = np.ascontiguousarray(seeds, np.int64)
        out = np.empty((self.V, len(s)), np.float64)
        lgo().lgo_ppr(self.h, level, _p(s), len(s), iterations, damping, _p(out))
        return out


class Reference(_Base):
    """The reference's own code compiled from source (oracle/_ref)."""

    def __init__(self, V):
        self.V = int(V)
        self.h = ref().llref_create(self.V)

    def __del__(self):
        if getattr(self, "h", None):
            ref().llref_destroy(self.h)
            self.h = None

    @staticmethod
    def set_threads(n):
        ref().llref_set_threads(int(n))

    @staticmethod
    def max_threads():
        return ref().llref_max_threads()

    @property
    def num_levels(self):
        return ref().llref_num_levels(self.h)

    def add_level(self, src, dst, del_src=(), del_dst=(), weights=None):
        s, d, ds, dd = _u32(src), _u32(dst), _u32(del_src), _u32(del_dst)
        order = np.lexsort((d, s))
        s, d = np.ascontiguousarray(s[order]), np.ascontiguousarray(d[order])
        if weights is None:
            r = ref().llref_add_level(self.h, _p(s), _p(d), len(s), _p(ds), _p(dd), len(ds))
        else:
            w = np.ascontiguousarray(_u32(weights)[order])
            r = ref().llref_add_level_weighted(self.h, _p(s), _p(d), len(s), _p(ds),
                                               _p(dd), len(ds), _p(w))
        if r != 0:
            raise ValueError(f"reference harness rejected the level ({r})")

    def sssp(self, level, root):
        out = np.empty(self.V, np.uint32)
        secs = ref().llref_sssp(self.h, level, int(root), _p(out))
        return out, secs

    def bc(self, level, sources):
        src = np.ascontiguousarray(sources, np.int64)
        out = np.empty(self.V, np.float32)
        secs = ref().llref_bc(self.h, level, _p(src), len(src), _p(out))
        return out, secs

    def tc_u(self):
        secs = _D()
        n = ref().llref_tc_u(self.h, C.byref(secs))
        return n, secs.value

    def tarjan_scc_seconds(self, level=-1):
        return ref().llref_tarjan_scc(self.h, level)

    def level_arrays(self, level, direction=0):
        n = ref().llref_level_arrays(self.h, direction, level, None, None)
        if n < 0:
            raise ValueError("no such level")
        vt = np.empty((self.V + 1) * 16, np.uint8)
        et = np.empty(max(n, 1), np.uint64)
        ref().llref_level_arrays(self.h, direction, level, _p(vt), _p(et))
        return vt.view(VT_DTYPE), et[:n]

    def adjacency(self, level, direction=0):
        off = np.empty(self.V + 1, np.uint64)
        n = ref().llref_adjacency(self.h, direction, level, _p(off), None)
        nb = np.empty(max(n, 1), np.uint32)
        ref().llref_adjacency(self.h, direction, level, _p(off), _p(nb))
        return off, nb[:n]

    def degrees(self, level):
        d = np.empty(self.V, np.uint32)
        ref().llref_degrees(self.h, level, _p(d))
        return d

    def pagerank_pull(self, level, iterations, damping=0.85):
        out = np.empty(self.V, np.float64)
        secs = ref().llref_pagerank(self.h, level, iterations, damping, _p(out))
        return out, secs

    def pagerank_push(self, level, iterations, damping=0.85):
        out = np.empty(self.V, np.float64)
        secs = ref().llref_pagerank_push(self.h, level, iterations, damping, _p(out))
        return out, secs

    def bfs(self, level, root):
        out = np.empty(self.V, np.int32)
        secs = ref().llref_bfs_levels(self.h, level, int(root), _p(out))
        return out, secs

    def bfs_count(self, level, root):
        secs = _D()
        cnt = ref().llref_bfs_count(self.h, level, int(root), C.byref(secs))
        return cnt, secs.value
