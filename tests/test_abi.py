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


def test_plain_c_program_builds_and_links(tmp_path):
    """A C99 host (what a cgo or other FFI stub compiles against) includes
    both headers with warnings as errors, links liblg.so and calls it: the
    version string, and a store that either opens (GPU present) or fails
    with LG_ECUDA and a message (no GPU), never a CPU fallback."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "host.c"
    src.write_text(
        '#include "lg.h"\n#include "lg_host.h"\n#include <stdio.h>\n'
        "int main(void) {\n"
        "  lg_store* s = NULL;\n"
        "  lg_store_opts o = {0};\n"
        "  lg_status st = lg_store_create(&s, &o);\n"
        "  printf(\"%s %d\\n\", lg_version(), (int)st);\n"
        "  if (st == LG_OK) return lg_store_destroy(s) == LG_OK ? 0 : 1;\n"
        "  char msg[256];\n"
        "  lg_last_error(msg, sizeof msg);\n"
        "  return (st == LG_ECUDA && msg[0] != 0) ? 0 : 2;\n"
        "}\n")
    exe = tmp_path / "host"
    libdir = os.path.dirname(lb.LIB_PATH)
    subprocess.check_call([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror",
                           "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                           "-L", libdir, "-llg", "-Wl,-rpath," + libdir])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.stdout, r.stderr)
    version, status = r.stdout.split()
    assert version == lb.lib.lg_version().decode()
    assert int(status) in (_lib.LG_OK, _lib.LG_ECUDA)
