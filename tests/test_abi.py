"""The C ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import glob
import os
import re

import pytest

import llama_b200 as lb
from llama_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(lg_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared()
    assert "lg_pagerank_pull" in names and "lg_store_create" in names
    missing = [n for n in sorted(names) if not hasattr(_lib.lib, n)]
    assert not missing, missing


def test_bindings_cover_every_declaration():
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert declared() <= bound, sorted(declared() - bound)


def test_version_and_status_strings():
    assert lb.lib.lg_version().decode().count(".") == 2
    assert lb.lib.lg_status_string(_lib.LG_EINVAL) == b"invalid argument"


def test_store_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lb.LgError) as e:
        lb.Store()
    assert e.value.status == _lib.LG_ECUDA
