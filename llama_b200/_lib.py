"""ctypes binding of liblg.so (include/lg.h, include/lg_host.h).

The library is built in-tree by ``make -C llama_b200`` (``__graft_entry__.build``)
and loaded from this package directory.  There is no fallback: if the shared
library is missing, importing the package raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblg.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C llama_b200` "
        "(or __graft_entry__.build()); llama_b200 has no CPU fallback")

lib = C.CDLL(LIB_PATH)

# ---------------------------------------------------------------- constants
LG_OK, LG_EINVAL, LG_ENOMEM, LG_ECUDA, LG_ETIMEOUT, LG_ESTATE, LG_ENOTSUP = range(7)
LG_BITS_LEVEL = 26
LG_BITS_INDEX = 38
LG_NIL_EDGE = -1
LG_FRESH_MAX_LEVEL = (1 << 26) - 1
LG_MAX_LEVELS = 64
LG_UNREACHED = 2147483646
LG_OUTPUT_SYNC = 0
LG_OUTPUT_ASYNC = 1
LG_ASYNC_MIN_BYTES = 1 << 20
LG_GEN_RMAT = 0
LG_GEN_KRONECKER = 1
LG_TUNE_PR_CTAS_PER_SM = 0
LG_TUNE_PPR_KTILE = 1
LG_TUNE_PPR_RANGE = 2
LG_TUNE_SSSP_RANGE = 3
LG_TUNE_MS_HEAVY = 4
LG_TUNE_PR_TILE_OCC = 5
LG_TUNE_SSSP_SPLIT = 6
LG_TUNE_BFS_LEVELS = 7
LG_TUNE_SSSP_LEVELS = 8
LG_TUNE_COUNT = 9
LG_TUNE_MAX_DEVICES = 64


class lg_vt_entry(C.Structure):
    _fields_ = [("adj_list_start", C.c_int64), ("level_length", C.c_uint32),
                ("degree", C.c_uint32)]


VT_DTYPE = np.dtype([("adj_list_start", "<i8"), ("level_length", "<u4"),
                     ("degree", "<u4")])


class lg_csr_level(C.Structure):
    _fields_ = [("max_nodes", C.c_uint64), ("vt", C.c_void_p),
                ("vt_pages", C.c_void_p), ("n_slots", C.c_uint64),
                ("slots", C.c_void_p), ("weights", C.c_void_p)]


class lg_deletion(C.Structure):
    _fields_ = [("edge", C.c_int64), ("max_visible_level", C.c_uint32),
                ("reserved", C.c_uint32)]


class lg_level_desc(C.Structure):
    _fields_ = [("out", lg_csr_level), ("in_", lg_csr_level),
                ("out_deletions", C.c_void_p), ("n_out_deletions", C.c_uint64),
                ("in_deletions", C.c_void_p), ("n_in_deletions", C.c_uint64)]


class lg_store_opts(C.Structure):
    _fields_ = [("device", C.c_int), ("stream", C.c_void_p),
                ("reverse_edges", C.c_int), ("reserved", C.c_int)]


class lg_bfs_result(C.Structure):
    _fields_ = [("reached", C.c_uint64), ("reach_edges", C.c_uint64),
                ("max_level", C.c_int32), ("top_down_steps", C.c_int32),
                ("bottom_up_steps", C.c_int32), ("reserved", C.c_int32)]


class lg_sssp_result(C.Structure):
    _fields_ = [("reached", C.c_uint64), ("reach_edges", C.c_uint64),
                ("max_dist", C.c_uint32), ("buckets", C.c_int32),
                ("rounds", C.c_int32), ("reserved", C.c_int32),
                ("relaxations", C.c_uint64)]


class lg_tc_result(C.Structure):
    _fields_ = [("triangles", C.c_int64), ("undirected_edges", C.c_uint64),
                ("arcs", C.c_uint64)]


class lg_teen_result(C.Structure):
    _fields_ = [("average", C.c_double), ("teen_sum", C.c_int64), ("vertices", C.c_int64)]


class lg_scc_result(C.Structure):
    _fields_ = [("components", C.c_uint64), ("trimmed", C.c_uint64),
                ("rounds", C.c_int32), ("steps", C.c_int32)]


class lg_fixed_point_result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("reserved", C.c_int32),
                ("residual", C.c_double)]


class lg_snapshot_stats(C.Structure):
    _fields_ = [("max_nodes", C.c_uint64), ("live_edges", C.c_uint64),
                ("slots", C.c_uint64), ("fragment_slots", C.c_uint64),
                ("fragments", C.c_uint64), ("ranges", C.c_uint64),
                ("deletions", C.c_uint64)]


class lg_tune_trial(C.Structure):
    _fields_ = [("key", C.c_int32), ("chosen", C.c_int32), ("value", C.c_int64),
                ("ms", C.c_double)]


class lg_graph_spec(C.Structure):
    _fields_ = [("kind", C.c_int), ("scale", C.c_int), ("edge_factor", C.c_double),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double),
                ("seed", C.c_uint64), ("symmetrize", C.c_int),
                ("num_levels", C.c_int), ("level0_fraction", C.c_double),
                ("delete_fraction", C.c_double), ("split_seed", C.c_uint64),
                ("weight_max", C.c_uint32), ("weight_seed", C.c_uint64)]


_P = C.c_void_p
_U64 = C.c_uint64
_I64 = C.c_int64
_INT = C.c_int
_D = C.c_double
_PP = C.POINTER(C.c_void_p)

# (name, restype, argtypes) for every entry point the headers declare.
SIGNATURES = [
    # lg.h
    ("lg_store_create", _INT, [_PP, C.POINTER(lg_store_opts)]),
    ("lg_store_destroy", _INT, [_P]),
    ("lg_store_ingest_level", _INT, [_P, C.POINTER(lg_level_desc)]),
    ("lg_store_num_levels", _INT, [_P]),
    ("lg_store_max_nodes", _INT, [_P, _INT, C.POINTER(_U64)]),
    ("lg_store_sync", _INT, [_P]),
    ("lg_store_set_output_mode", _INT, [_P, _INT]),
    ("lg_store_stream", _P, [_P]),
    ("lg_store_device_bytes", _U64, [_P]),
    ("lg_store_launch_count", _U64, [_P]),
    ("lg_store_transfer_bytes", _INT, [_P, C.POINTER(_U64), C.POINTER(_U64)]),
    ("lg_store_drop_level", _INT, [_P]),
    ("lg_store_build_level", _INT, [_P, _U64, _P, _P, _P, _U64, _P, _P, _U64]),
    ("lg_store_read_level", _INT, [_P, _INT, _INT, _P, _P, _P, C.POINTER(_U64)]),
    ("lg_snapshot_get_stats", _INT, [_P, _INT, C.POINTER(lg_snapshot_stats)]),
    ("lg_snapshot_open", _INT, [_P, _INT, _PP]),
    ("lg_snapshot_open_window", _INT, [_P, _INT, _INT, _PP]),
    ("lg_snapshot_min_level", _INT, [_P, C.POINTER(_INT)]),
    ("lg_store_set_min_level", _INT, [_P, _INT]),
    ("lg_store_min_level", _INT, [_P]),
    ("lg_snapshot_close", _INT, [_P]),
    ("lg_snapshot_level", _INT, [_P, C.POINTER(_INT)]),
    ("lg_snapshot_max_nodes", _INT, [_P, C.POINTER(_U64)]),
    ("lg_snapshot_num_edges", _INT, [_P, C.POINTER(_U64)]),
    ("lg_out_degrees", _INT, [_P, _P]),
    ("lg_in_degrees", _INT, [_P, _P]),
    ("lg_snapshot_adjacency", _INT, [_P, _INT, _P, _P, _P]),
    ("lg_snapshot_flatten", _INT, [_P, _INT]),
    ("lg_snapshot_unflatten", _INT, [_P]),
    ("lg_snapshot_is_flat", _INT, [_P, _INT, C.POINTER(_INT)]),
    ("lg_pagerank_pull", _INT, [_P, _INT, _D, _P]),
    ("lg_pagerank_push", _INT, [_P, _INT, _D, _P]),
    ("lg_pagerank_pull_noalloc", _INT, [_P, _INT, _D, _P]),
    ("lg_pagerank_gather_pass", _INT, [_P, _INT, C.POINTER(_D)]),
    ("lg_bfs", _INT, [_P, _I64, _P, C.POINTER(lg_bfs_result)]),
    ("lg_bfs_multi", _INT, [_P, _P, _INT, _P, _P]),
    ("lg_sssp_delta", _INT, [_P, _I64, C.c_uint32, _P, C.POINTER(lg_sssp_result)]),
    ("lg_triangle_count", _INT, [_P, C.POINTER(lg_tc_result)]),
    ("lg_avg_teen_cnt", _INT, [_P, _P, _INT, _P, C.POINTER(lg_teen_result)]),
    ("lg_scc", _INT, [_P, _P, C.POINTER(lg_scc_result)]),
    ("lg_bc", _INT, [_P, _P, _INT, _P]),
    ("lg_bc_batched", _INT, [_P, _P, _INT, _P]),
    ("lg_ppr", _INT, [_P, _INT, _P, _INT, _INT, _D, _P]),
    ("lg_pagerank_fwd", _INT, [_P, _P, _P, _D, _D, _INT, _P, _PP,
                               C.POINTER(lg_fixed_point_result)]),
    ("lg_pagerank_bwd", _INT, [_P, _P, _P, _P, C.POINTER(lg_fixed_point_result)]),
    ("lg_adjoint_free", _INT, [_P]),
    ("lg_tune_get", _INT, [_INT, _INT, C.POINTER(_I64)]),
    ("lg_tune_set", _INT, [_INT, _INT, _I64]),
    ("lg_tune_reset", _INT, [_INT]),
    ("lg_autotune", _INT, [_P, C.c_uint, C.POINTER(lg_tune_trial), _INT, C.POINTER(_INT)]),
    ("lg_last_error", C.c_size_t, [C.c_char_p, C.c_size_t]),
    ("lg_status_string", C.c_char_p, [_INT]),
    ("lg_version", C.c_char_p, []),
    # lg_host.h
    ("lg_hgraph_create", _INT, [_PP, _U64, _INT]),
    ("lg_hgraph_destroy", _INT, [_P]),
    ("lg_hgraph_add_level", _INT, [_P, _P, _P, _U64, _P, _P, _U64, _P]),
    ("lg_hgraph_num_levels", _INT, [_P]),
    ("lg_hgraph_max_nodes", _U64, [_P]),
    ("lg_hgraph_level_desc", _INT, [_P, _INT, C.POINTER(lg_level_desc)]),
    ("lg_hgraph_ingest", _INT, [_P, _P, _INT]),
    ("lg_hgraph_level_input", _INT, [_P, _INT, _PP, _PP, C.POINTER(_U64), _PP,
                                     _PP, C.POINTER(_U64), _PP]),
    ("lg_gen_edges", _INT, [C.POINTER(lg_graph_spec), _P, _P, _U64, C.POINTER(_U64)]),
    ("lg_hgraph_build", _INT, [_P, C.POINTER(lg_graph_spec)]),
    ("lg_gen_weight", C.c_uint32, [C.POINTER(lg_graph_spec), C.c_uint32, C.c_uint32]),
]

for _name, _res, _args in SIGNATURES:
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class LgError(RuntimeError):
    """A non-zero lg_status, with the library's message."""

    def __init__(self, status, message):
        super().__init__(f"{lib.lg_status_string(status).decode()} ({status}): {message}")
        self.status = status
        self.message = message


def last_error():
    buf = C.create_string_buffer(1024)
    lib.lg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != LG_OK:
        raise LgError(status, last_error())
    return status


def ptr(x):
    """Address of a numpy array, a torch tensor, or None."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return x.ctypes.data
    if isinstance(x, int):
        return x
    raise TypeError(f"cannot take the address of {type(x)}")
