"""bench.py's host-side contract, on CPU.

The reference arm must build its inputs without the engine (its process must
never map liblg.so) and report the same config as the device arm; the
workload parameters bench.py passes around as plain values must be the ones
llama_b200.workloads builds the device arm's graphs from."""
import json
import os
import subprocess
import sys

import pytest

import bench
from llama_b200 import workloads
from llama_b200.graph import GraphSpec
from oracle.bind import ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def fields(spec):
    return {k: getattr(spec, k) for k in GraphSpec.__dataclass_fields__}


def test_workload_params_match_the_engine_workloads():
    assert bench.rmat_params(24, 2, 8, 0.90, 0.002, weight_max=255) == fields(
        workloads.rmat_multiversion(scale=24, seed=2, levels=8, level0=0.90, delete=0.002,
                                    weight_max=255))
    assert bench.kron_params(21, 6, 4) == fields(
        workloads.kronecker_symmetric(scale=21, seed=6, levels=4))


def test_max_rel():
    assert bench.max_rel([0.0, 1.0], [0.0, 1.0]) == 0.0
    assert bench.max_rel([1.0 + 1e-9], [1.0]) == pytest.approx(1e-9, rel=1e-3)
    assert bench.max_rel([1e-300], [0.0]) == 1.0


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_arm_runs_without_the_engine():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--scale", "11", "--levels", "3", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["engine_loaded"] is False
    assert line["unit"] == "GTEPS" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # the config is the device arm's for the same flags
    sys_argv = sys.argv
    try:
        sys.argv = ["bench.py", "--scale", "11", "--levels", "3"]
        args = bench.parse()
    finally:
        sys.argv = sys_argv
    assert line["config"] == bench.workload(args)[1]
