"""Python mirror of the LLAMA analytics interface over liblg.

Names follow the reference: a ``HostGraph`` plays the writable side that
checkpoints levels (``ll_writable_graph::checkpoint``), a ``Store`` the
``ll_database`` that owns the read-only level stack, a ``Snapshot`` the view
``ll_mlcsr_ro_graph(master, level)``, and the analytics methods are the
benchmark tasks of ``benchmark -r <task>`` (benchmark/benchmark.cc:871-946).
Every call goes through the C ABI in include/lg.h; results come back as numpy
arrays, or are written into caller-provided torch CUDA tensors.
"""
import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from ._lib import check, lib, ptr


@dataclass
class GraphSpec:
    """Seeded synthetic multiversion graph (``lg_graph_spec``)."""
    scale: int
    edge_factor: float = 16.0
    a: float = 0.57
    b: float = 0.19
    c: float = 0.19
    seed: int = 1
    kind: int = _lib.LG_GEN_RMAT
    symmetrize: bool = False
    num_levels: int = 1
    level0_fraction: float = 1.0
    delete_fraction: float = 0.0
    split_seed: int = 0
    weight_max: int = 0
    weight_seed: int = 0

    def to_c(self):
        s = _lib.lg_graph_spec()
        for f in fields(self):
            setattr(s, f.name, int(getattr(self, f.name))
                    if isinstance(getattr(self, f.name), bool) else getattr(self, f.name))
        return s

    @property
    def max_nodes(self):
        return 1 << self.scale


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class HostGraph:
    """Host-side multiversion graph in the reference's level layout."""

    def __init__(self, max_nodes, reverse_edges=True):
        h = C.c_void_p()
        check(lib.lg_hgraph_create(C.byref(h), int(max_nodes), int(bool(reverse_edges))))
        self._h = h
        self.max_nodes = int(max_nodes)
        self.reverse_edges = bool(reverse_edges)

    @classmethod
    def from_spec(cls, spec, reverse_edges=True):
        g = cls(spec.max_nodes, reverse_edges)
        check(lib.lg_hgraph_build(g._h, C.byref(spec.to_c())))
        return g

    def close(self):
        if self._h:
            lib.lg_hgraph_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h

    @property
    def num_levels(self):
        return lib.lg_hgraph_num_levels(self._h)

    def add_level(self, src, dst, del_src=(), del_dst=(), weights=None):
        src, dst = _u32(src), _u32(dst)
        ds, dd = _u32(del_src), _u32(del_dst)
        w = None if weights is None else _u32(weights)
        check(lib.lg_hgraph_add_level(self._h, ptr(src), ptr(dst), len(src),
                                      ptr(ds), ptr(dd), len(ds), ptr(w)))

    def level_input(self, level):
        """(src, dst, del_src, del_dst, weights) the level was built from."""
        ps, pd, pds, pdd, pw = (C.c_void_p() for _ in range(5))
        n, nd = C.c_uint64(), C.c_uint64()
        check(lib.lg_hgraph_level_input(self._h, level, C.byref(ps), C.byref(pd),
                                        C.byref(n), C.byref(pds), C.byref(pdd),
                                        C.byref(nd), C.byref(pw)))

        def arr(p, k):
            if k == 0 or not p.value:
                return np.zeros(0, np.uint32)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), (k,)).copy()
        w = arr(pw, n.value) if pw.value else None
        return (arr(ps, n.value), arr(pd, n.value), arr(pds, nd.value),
                arr(pdd, nd.value), w)

    def level_desc(self, level):
        d = _lib.lg_level_desc()
        check(lib.lg_hgraph_level_desc(self._h, level, C.byref(d)))
        return d

    def level_arrays(self, level, direction=0):
        """(vertex table, slots) of one level as numpy copies."""
        d = self.level_desc(level)
        c = d.out if direction == 0 else d.in_
        vt = np.ctypeslib.as_array(C.cast(c.vt, C.POINTER(C.c_uint8)),
                                   ((c.max_nodes + 1) * 16,)).copy().view(_lib.VT_DTYPE)
        if c.n_slots:
            sl = np.ctypeslib.as_array(C.cast(c.slots, C.POINTER(C.c_uint64)),
                                       (c.n_slots,)).copy()
        else:
            sl = np.zeros(0, np.uint64)
        return vt, sl


class Store:
    """Device mirror of the level stack (``lg_store``)."""

    def __init__(self, device=0, stream=None, reverse_edges=True):
        o = _lib.lg_store_opts(device=device, stream=stream or None,
                               reverse_edges=int(bool(reverse_edges)))
        h = C.c_void_p()
        check(lib.lg_store_create(C.byref(h), C.byref(o)))
        self._h = h
        self.reverse_edges = bool(reverse_edges)

    def close(self):
        if self._h:
            check(lib.lg_store_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def num_levels(self):
        return lib.lg_store_num_levels(self._h)

    @property
    def stream(self):
        return lib.lg_store_stream(self._h)

    @property
    def device_bytes(self):
        return lib.lg_store_device_bytes(self._h)

    def ingest(self, hgraph, first=None):
        first = self.num_levels if first is None else first
        check(lib.lg_hgraph_ingest(hgraph.handle, self._h, first))

    def ingest_level(self, desc):
        check(lib.lg_store_ingest_level(self._h, C.byref(desc)))

    def sync(self):
        check(lib.lg_store_sync(self._h))

    def set_output_mode(self, mode):
        """"sync" (default) or "async": with "async", results of 1 MiB or more
        written to page-locked host tensors are copied on a second stream and
        are in place after sync() (lg_store_set_output_mode)."""
        m = {"sync": _lib.LG_OUTPUT_SYNC, "async": _lib.LG_OUTPUT_ASYNC}.get(mode, mode)
        check(lib.lg_store_set_output_mode(self._h, int(m)))

    @property
    def launch_count(self):
        return lib.lg_store_launch_count(self._h)

    def drop_level(self):
        check(lib.lg_store_drop_level(self._h))

    def transfer_bytes(self):
        """(host->device, device->host) bytes copied by this store so far."""
        h, d = C.c_uint64(), C.c_uint64()
        check(lib.lg_store_transfer_bytes(self._h, C.byref(h), C.byref(d)))
        return h.value, d.value

    def build_level(self, max_nodes, src, dst, weights=None, del_src=(), del_dst=()):
        """Build the next level on the device from its edge delta
        (``lg_store_build_level``).  Arrays may be numpy (host) or torch CUDA
        tensors of uint32/int32."""
        def arr(a):
            if hasattr(a, "data_ptr"):
                return a, a.numel()
            a = _u32(a)
            return a, len(a)
        s, n = arr(src)
        d, _ = arr(dst)
        ds, nd = arr(del_src)
        dd, _ = arr(del_dst)
        w = None if weights is None else arr(weights)[0]
        check(lib.lg_store_build_level(self._h, int(max_nodes), ptr(s), ptr(d), ptr(w), n,
                                       ptr(ds) if nd else None, ptr(dd) if nd else None, nd))

    def read_level(self, level, direction=0, weights=False):
        """(vertex table, ids[, weights]) of a level as the device holds it."""
        n = C.c_uint64()
        check(lib.lg_store_read_level(self._h, level, direction, None, None, None, C.byref(n)))
        mn = C.c_uint64()
        check(lib.lg_store_max_nodes(self._h, level, C.byref(mn)))
        vt = np.empty(mn.value + 1, _lib.VT_DTYPE)
        ids = np.empty(max(n.value, 1), np.uint32)
        w = np.empty(max(n.value, 1), np.uint32) if weights else None
        check(lib.lg_store_read_level(self._h, level, direction, ptr(vt), ptr(ids), ptr(w),
                                      None))
        ids = ids[:n.value]
        if weights:
            return vt, ids, w[:n.value]
        return vt, ids

    def snapshot(self, level=-1, min_level=None):
        """Snapshot of `level`; with min_level, a sliding window over levels
        min_level..level."""
        return Snapshot(self, level, min_level)

    @property
    def min_level(self):
        return lib.lg_store_min_level(self._h)

    def set_min_level(self, m):
        """Age out the levels below m (lg_store_set_min_level)."""
        check(lib.lg_store_set_min_level(self._h, int(m)))


class Tape:
    """Converged scores of a lg_pagerank_fwd call, for lg_pagerank_bwd."""

    def __init__(self, handle, snapshot):
        self._h = handle
        self.snapshot = snapshot

    def backward(self, dldx, dldw=None, dldv=None):
        """Returns (dL/dweights, dL/dteleport, result)."""
        g = np.ascontiguousarray(dldx, np.float64) if not hasattr(dldx, "data_ptr") else dldx
        if dldw is None:
            dldw = np.empty(self.snapshot.num_edges, np.float64)
        if dldv is None:
            dldv = np.empty(self.snapshot.max_nodes, np.float64)
        r = _lib.lg_fixed_point_result()
        check(lib.lg_pagerank_bwd(self._h, ptr(g), ptr(dldw), ptr(dldv), C.byref(r)))
        return dldw, dldv, r

    def close(self):
        if self._h:
            lib.lg_adjoint_free(self._h)
            self._h = None

    __del__ = close


TUNABLES = {"pr_ctas_per_sm": _lib.LG_TUNE_PR_CTAS_PER_SM,
            "ppr_ktile": _lib.LG_TUNE_PPR_KTILE,
            "ppr_range": _lib.LG_TUNE_PPR_RANGE,
            "sssp_range": _lib.LG_TUNE_SSSP_RANGE,
            "ms_heavy": _lib.LG_TUNE_MS_HEAVY,
            "pr_tile_occ": _lib.LG_TUNE_PR_TILE_OCC,
            "sssp_split": _lib.LG_TUNE_SSSP_SPLIT,
            "bfs_levels": _lib.LG_TUNE_BFS_LEVELS,
            "sssp_levels": _lib.LG_TUNE_SSSP_LEVELS}


def tune_set(device, name, value):
    """Pin launch parameter `name` (a TUNABLES key) of a GPU (lg_tune_set)."""
    check(lib.lg_tune_set(int(device), TUNABLES[name], int(value)))


def tune_get(device, name):
    v = C.c_int64()
    check(lib.lg_tune_get(int(device), TUNABLES[name], C.byref(v)))
    return v.value


def tune_reset(device):
    check(lib.lg_tune_reset(int(device)))


def ppr(snapshots, seeds, iterations=20, damping=0.85, out=None):
    """Personalized PageRank (``lg_ppr``) for len(seeds) seeds on every
    snapshot in one captured graph; returns [n_snaps, max_nodes, K]."""
    snaps = list(snapshots)
    arr = (C.c_void_p * len(snaps))(*[s.handle.value for s in snaps])
    s = np.ascontiguousarray(seeds, np.int64)
    V = snaps[0].max_nodes
    res = np.empty((len(snaps), V, len(s)), np.float64) if out is None else out
    check(lib.lg_ppr(C.cast(arr, C.c_void_p), len(snaps), ptr(s), len(s), int(iterations),
                     float(damping), ptr(res)))
    return res


class Snapshot:
    """Read-only view of one level (``lg_snapshot``)."""

    def __init__(self, store, level=-1, min_level=None):
        h = C.c_void_p()
        if min_level is None:
            check(lib.lg_snapshot_open(store.handle, level, C.byref(h)))
        else:
            check(lib.lg_snapshot_open_window(store.handle, level, int(min_level), C.byref(h)))
        self._h = h
        self.store = store
        lv, mn, ml = C.c_int(), C.c_uint64(), C.c_int()
        check(lib.lg_snapshot_level(h, C.byref(lv)))
        check(lib.lg_snapshot_max_nodes(h, C.byref(mn)))
        check(lib.lg_snapshot_min_level(h, C.byref(ml)))
        self.level = lv.value
        self.max_nodes = mn.value
        self.min_level = ml.value

    def close(self):
        if self._h:
            check(lib.lg_snapshot_close(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def num_edges(self):
        n = C.c_uint64()
        check(lib.lg_snapshot_num_edges(self._h, C.byref(n)))
        return n.value

    def stats(self, direction=0):
        st = _lib.lg_snapshot_stats()
        check(lib.lg_snapshot_get_stats(self._h, direction, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def out_degrees(self):
        out = np.empty(self.max_nodes, np.uint32)
        check(lib.lg_out_degrees(self._h, ptr(out)))
        return out

    def in_degrees(self):
        out = np.empty(self.max_nodes, np.uint32)
        check(lib.lg_in_degrees(self._h, ptr(out)))
        return out

    def adjacency(self, direction=0, with_edge_ids=False):
        """(offsets, neighbours[, edge ids]) in the reference's iteration order."""
        off = np.empty(self.max_nodes + 1, np.uint64)
        check(lib.lg_snapshot_adjacency(self._h, direction, ptr(off), None, None))
        n = int(off[-1])
        nb = np.empty(max(n, 1), np.uint32)
        ei = np.empty(max(n, 1), np.int64) if with_edge_ids else None
        check(lib.lg_snapshot_adjacency(self._h, direction, ptr(off), ptr(nb), ptr(ei)))
        if with_edge_ids:
            return off, nb[:n], ei[:n]
        return off, nb[:n]

    def flatten(self, direction=1):
        """Keep direction `direction` (0 out, 1 in) as one flat CSR on the
        device; traversals of it on this snapshot read that instead."""
        check(lib.lg_snapshot_flatten(self._h, int(direction)))
        return self

    def unflatten(self):
        check(lib.lg_snapshot_unflatten(self._h))
        return self

    def is_flat(self, direction=1):
        f = C.c_int()
        check(lib.lg_snapshot_is_flat(self._h, int(direction), C.byref(f)))
        return bool(f.value)

    # ---- benchmark tasks -------------------------------------------------
    def pagerank_pull(self, iterations=10, damping=0.85, out=None):
        """Task ``pagerank_double``: FP64 pull PageRank."""
        res = np.empty(self.max_nodes, np.float64) if out is None else out
        check(lib.lg_pagerank_pull(self._h, int(iterations), float(damping), ptr(res)))
        return res

    def pagerank_push(self, iterations=10, damping=0.85, out=None):
        """Task ``pagerank_double_push``: FP64 push PageRank over the out-CSR."""
        res = np.empty(self.max_nodes, np.float64) if out is None else out
        check(lib.lg_pagerank_push(self._h, int(iterations), float(damping), ptr(res)))
        return res

    def bfs(self, root, out=None):
        """Task ``sssp_unweighted`` (BFS levels); returns (levels, lg_bfs_result)."""
        res = np.empty(self.max_nodes, np.int32) if out is None else out
        r = _lib.lg_bfs_result()
        check(lib.lg_bfs(self._h, int(root), ptr(res), C.byref(r)))
        return res, r

    def bfs_multi(self, roots, out=None):
        """BFS levels from every root in one call: (levels[n][V], results)."""
        r = np.ascontiguousarray(roots, dtype=np.int64)
        res = np.empty((len(r), self.max_nodes), np.int32) if out is None else out
        rs = (_lib.lg_bfs_result * len(r))()
        check(lib.lg_bfs_multi(self._h, ptr(r), len(r), ptr(res), rs))
        return res, list(rs)

    def scc(self, out=None):
        """Strongly connected components, labelled by their smallest vertex;
        returns (labels, lg_scc_result)."""
        res = np.empty(self.max_nodes, np.int64) if out is None else out
        r = _lib.lg_scc_result()
        check(lib.lg_scc(self._h, ptr(res), C.byref(r)))
        return res, r

    def bc(self, sources, batched=True, out=None):
        """Brandes BC from `sources` (FP64); batched = 64 sources per pass."""
        src = np.ascontiguousarray(sources, np.int64)
        res = np.empty(self.max_nodes, np.float64) if out is None else out
        fn = lib.lg_bc_batched if batched else lib.lg_bc
        check(fn(self._h, ptr(src), len(src), ptr(res)))
        return res

    def gather_pass(self, passes=1):
        """`passes` passes of the PageRank iteration's loads alone over the
        flat in-CSR (``lg_pagerank_gather_pass``); returns the checksum."""
        c = C.c_double()
        check(lib.lg_pagerank_gather_pass(self._h, int(passes), C.byref(c)))
        return c.value

    def gather_pass_async(self, passes=1):
        """The same without reading the checksum back (for timing)."""
        check(lib.lg_pagerank_gather_pass(self._h, int(passes), None))

    def autotune(self, names=None):
        """Measure the launch parameters `names` (TUNABLES keys, default all)
        on this snapshot and keep the fastest (``lg_autotune``); returns
        {name: {"chosen": value, "ms": {value: median ms}}}."""
        names = list(TUNABLES) if names is None else list(names)
        mask = 0
        for n in names:
            mask |= 1 << TUNABLES[n]
        trials = (_lib.lg_tune_trial * 64)()
        count = C.c_int()
        check(lib.lg_autotune(self._h, mask, trials, 64, C.byref(count)))
        by_key = {v: k for k, v in TUNABLES.items()}
        out = {}
        for t in trials[:count.value]:
            d = out.setdefault(by_key[t.key], {"chosen": None, "ms": {}})
            d["ms"][int(t.value)] = t.ms
            if t.chosen:
                d["chosen"] = int(t.value)
        return out

    def pagerank_fwd(self, weights, teleport, damping=0.85, tol=1e-12, max_iter=10000,
                     keep_tape=True, out=None):
        """Weighted PageRank fixed point (``lg_pagerank_fwd``); weights follow
        the out-adjacency order.  Returns (x, Tape or None, result)."""
        w = np.ascontiguousarray(weights, np.float64) if not hasattr(weights, "data_ptr") else weights
        v = np.ascontiguousarray(teleport, np.float64) if not hasattr(teleport, "data_ptr") else teleport
        x = np.empty(self.max_nodes, np.float64) if out is None else out
        t = C.c_void_p()
        r = _lib.lg_fixed_point_result()
        check(lib.lg_pagerank_fwd(self._h, ptr(w), ptr(v), float(damping), float(tol),
                                  int(max_iter), ptr(x), C.byref(t) if keep_tape else None,
                                  C.byref(r)))
        return x, (Tape(t, self) if keep_tape else None), r

    def triangle_count(self):
        """Task ``tc_u`` on the symmetrised snapshot; returns lg_tc_result."""
        r = _lib.lg_tc_result()
        check(lib.lg_triangle_count(self._h, C.byref(r)))
        return r

    def avg_teen_cnt(self, age, K=0, out=None):
        """Task ``avg_teen_cnt``: (teen_cnt per vertex, lg_teen_result).  age:
        int32 per vertex (numpy or a torch CUDA tensor)."""
        a = age if hasattr(age, "data_ptr") else np.ascontiguousarray(age, dtype=np.int32)
        res = np.empty(self.max_nodes, np.int32) if out is None else out
        r = _lib.lg_teen_result()
        check(lib.lg_avg_teen_cnt(self._h, ptr(a), int(K), ptr(res), C.byref(r)))
        return res, r

    def sssp(self, root, delta=32, out=None):
        """Task ``sssp_weighted`` (delta-stepping); returns (dist, lg_sssp_result)."""
        res = np.empty(self.max_nodes, np.uint32) if out is None else out
        r = _lib.lg_sssp_result()
        check(lib.lg_sssp_delta(self._h, int(root), int(delta), ptr(res), C.byref(r)))
        return res, r
