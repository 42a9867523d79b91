"""llama_b200 - B200-native analytics over LLAMA multiversioned CSR stores.

The engine is liblg.so (hand-written sm_100a CUDA behind the C ABI in
include/lg.h); this package is its Python mirror of the reference's
database / snapshot / benchmark-task interface.
"""
from ._lib import LG_UNREACHED, LgError, lib, LIB_PATH  # noqa: F401  (raises if not built)
from .graph import GraphSpec, HostGraph, Snapshot, Store  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["GraphSpec", "HostGraph", "Store", "Snapshot", "LgError", "workloads"]
