"""The N > 1 path of bench.py on CPU ranks (gloo, world size 2): replicas
report the slowest rank's time and all ranks' work, and the reference arm
runs on rank 0 alone while the other ranks leave without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench

    class Args:
        impl = "reference"      # gloo, as the reference arm uses

    w, r, _ = bench.dist_init(Args)
    bench.barrier(w)
    ms, edges = bench.reduce_max_sum(w, 10.0 * (r + 1), 100 * (r + 1))
    q.put((r, w, ms, edges))
    bench.barrier(w)
    dist.destroy_process_group()


def test_replicas_take_max_time_and_sum_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(o[0] for o in out) == [0, 1]
    for _, w, ms, edges in out:
        assert w == 2 and ms == 20.0 and edges == 300.0


def test_reference_arm_runs_on_rank_zero_only():
    from oracle.bind import ref_available
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", "bench.py",
           "--impl", "reference", "--scale", "10", "--levels", "3", "--steps", "1",
           "--warmup", "1", "--gpus", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
