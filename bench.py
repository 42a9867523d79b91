#!/usr/bin/env python
"""Benchmark: PageRank pull + BFS GTEPS over a multiversion R-MAT store.

Workload (default): directed R-MAT scale 24 (2^24 vertices, 16 * 2^24 draws,
a/b/c/d = .57/.19/.19/.05, self-loops and duplicates removed, seed 2), split
into 8 levels: a seeded 90 % of the edges form level 0, levels 1..7 each add
~1.4 % and delete 0.2 % of the live edges (deletion marks in older levels).
One step on the latest snapshot = flatten its in-CSR (lg_snapshot_flatten)
+ FP64 PageRank pull, 20 iterations, d = 0.85 + BFS from 16 roots (seed 3,
out-degree > 0) + free the flat CSR.

value    = traversed edges per second of the device-resident step:
           (20 * E_live + sum over roots of E_reach) / step time  [GTEPS]
e2e      = the same step through the C ABI with host buffers: every step
           rebuilds the newest level on the device from its edge delta in
           pinned host memory, reopens the snapshot and copies the ranks and
           BFS levels back to pinned host memory (on the store's copy
           stream, overlapped with the following work; all copies inside the
           timed region)
roofline = the PageRank iteration kernel (pr_flat_step), HBM-bound
bfs_roofline = the BFS phase against the per-root byte model (effective
           bandwidth; the multi-source roots share one traversal)
--impl reference times the reference's own OpenMP kernels (oracle/_ref, built
from the reference source) on the host cores for the same step.

N > 1 (torchrun): independent replicas, one store per GPU (the path does not
shard), weak scaling; value = all ranks' edges / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS (PageRank iter, BFS) on multiversion R-MAT; batched BC & adjoint vs plain"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="lg", choices=["lg", "reference"])
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--levels", type=int, default=8)
    p.add_argument("--pr-iters", type=int, default=20)
    p.add_argument("--roots", type=int, default=16)
    p.add_argument("--bfs", default="multi", choices=["multi", "single"],
                   help="BFS from all roots in one lg_bfs_multi call, or one lg_bfs per root")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the secondary kernels (SSSP, TC, SCC, BC, PPR, adjoint)")
    p.add_argument("--kron-scale", type=int, default=21)
    p.add_argument("--bc-sources", type=int, default=4096,
                   help="sources of the batched BC run (64 per pass)")
    p.add_argument("--adjoint-scale", type=int, default=20)
    p.add_argument("--out", default=None, help="also write the JSON line here")
    return p.parse_args()


def workload(args):
    from llama_b200 import workloads
    spec = workloads.rmat_multiversion(scale=args.scale, seed=2, levels=args.levels,
                                       level0=0.90, delete=0.002, weight_max=255)
    cfg = {"workload": f"rmat{args.scale}_{args.levels}level_del0.2pct",
           "graph": f"directed R-MAT scale {args.scale}, edge factor 16, "
                    f"{args.levels} levels (90% in level 0, 0.2% deletions per level)",
           "step": f"flatten the in-CSR + PageRank pull FP64 x{args.pr_iters} iterations "
                   f"+ BFS from {args.roots} roots, latest snapshot",
           "bfs_mode": ("all roots in one multi-source call (lg_bfs_multi, 64 roots per "
                        "bit-parallel pass; each row equals a single-root BFS)"
                        if args.bfs == "multi" else "one lg_bfs call per root"),
           "pr_iterations": args.pr_iters, "damping": 0.85, "bfs_roots": args.roots}
    return spec, cfg


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "lg" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


class Clocks:
    """SM clock and clock-event reasons sampled during the timed region: an
    NVML thread every 10 ms (device found by its PCI bus id), else
    nvidia-smi every 200 ms."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((mhz, self.max_mhz) +
                                     tuple("active" if r & b else "" for b in bits))
                    self.stop_flag.wait(0.01)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        rows, source = self.rows, "nvml 10 ms"
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
        elif self.p is not None:
            source = "nvidia-smi 200 ms"
            self.p.terminate()
            out, _ = self.p.communicate(timeout=10)
            for line in out.strip().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) < 8:
                    continue
                try:
                    rows.append((float(f[0]), float(f[1]), f[4], f[5], f[6], f[7]))
                except ValueError:
                    continue
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for name, v in zip(self.NAMES, r[2:]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "samples": len(rows),
                "source": source, "reasons": sorted(reasons)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per pr_flat_step launch at this workload, from the line
    `traffic_bytes_per_launch: N` of the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "pr_flat_step_rmat24.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return {"dram_bytes_per_launch_scaled": float(line.split(":")[1])}
    except (OSError, ValueError):
        pass
    return None


def run_reference(args):
    ws, rank, local = dist_init(args)
    if rank != 0:
        return
    from llama_b200 import HostGraph
    from oracle.bind import Reference, ref_available
    spec, cfg = workload(args)
    if not ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libllref.so was not built"}))
        return
    hg = HostGraph.from_spec(spec)
    R = Reference(spec.max_nodes)
    for l in range(hg.num_levels):
        R.add_level(*hg.level_input(l)[:4])
    del hg
    from llama_b200 import workloads
    deg = R.degrees(-1)
    roots = workloads.pick_roots(deg, args.roots, seed=3)
    E = int(deg.sum())
    cores = Reference.max_threads()

    # each step is a quarter of the device step, in the same proportions:
    # pr_iters/4 PageRank iterations + BFS from a quarter of the roots, the
    # roots taken in turn so that four steps cover all of them
    q_it = max(1, args.pr_iters // 4)
    q_roots = max(1, len(roots) // 4)

    def step(i):
        pr, t_pr = R.pagerank_pull(-1, q_it, 0.85)
        edges, t_bfs = 0, 0.0
        for j in range(q_roots):
            r = roots[(i * q_roots + j) % len(roots)]
            lv, t = R.bfs(-1, int(r))
            t_bfs += t
            edges += int(deg[lv < 2147483646].sum(dtype=np.int64))
        return t_pr + t_bfs, q_it * E + edges

    for i in range(args.warmup):
        step(i)
    tot_t, tot_e = 0.0, 0
    for i in range(args.steps):
        t, e = step(i)
        tot_t += t
        tot_e += e
    gteps = tot_e / tot_t / 1e9
    line = {"metric": METRIC, "value": gteps, "unit": "GTEPS", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": cores,
                             "kind": "reference",
                             "sample": f"each step = a quarter of the device step: "
                                       f"pagerank_double x{q_it} + sssp_unweighted BFS "
                                       f"from {q_roots} of the {len(roots)} roots in turn, "
                                       "on the same store, run() time only"},
            "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    emit(line, args)


def emit(line, args):
    s = json.dumps(line)
    print(s, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(s + "\n")


def run_lg(args):
    import torch
    ws, rank, local = dist_init(args)
    torch.cuda.set_device(local)
    from llama_b200 import HostGraph, Store, workloads
    spec, cfg = workload(args)
    cfg["parallelism"] = f"replicas{ws}"
    t0 = time.time()
    hg = HostGraph.from_spec(spec)
    build_s = time.time() - t0

    stream = torch.cuda.Stream(device=local)
    st = Store(device=local, stream=stream.cuda_stream)
    t0 = time.time()
    st.ingest(hg)
    ingest_s = time.time() - t0
    sn = st.snapshot()
    V = sn.max_nodes
    deg = sn.out_degrees()
    roots = workloads.pick_roots(deg, args.roots, seed=3)
    E = sn.num_edges
    ins = sn.stats(1)

    pr_dev = torch.empty(V, dtype=torch.float64, device=f"cuda:{local}")
    lv_dev = torch.empty((len(roots), V), dtype=torch.int32, device=f"cuda:{local}")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def step():
        # the in-CSR is flattened inside every step, used by PageRank and the
        # BFS bottom-up steps, and freed at the end of the step
        ev[0].record(stream)
        sn.flatten(1)
        ev[3].record(stream)
        sn.pagerank_pull(args.pr_iters, 0.85, out=pr_dev)
        ev[1].record(stream)
        reach = 0
        if args.bfs == "multi":
            _, rs = sn.bfs_multi(roots, out=lv_dev)
            reach = sum(r.reach_edges for r in rs)
        else:
            for i, r in enumerate(roots):
                _, res = sn.bfs(int(r), out=lv_dev[i])
                reach += res.reach_edges
        ev[2].record(stream)
        sn.unflatten()
        return reach

    for _ in range(max(3, args.warmup)):
        reach = step()
    st.sync()
    barrier(ws)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    launches0 = st.launch_count
    pr_ms, bfs_ms, flat_ms, edges = 0.0, 0.0, 0.0, 0
    t_start.record(stream)
    for _ in range(args.steps):
        reach = step()
        stream.synchronize()
        pr_ms += ev[0].elapsed_time(ev[1])
        flat_ms += ev[0].elapsed_time(ev[3])
        bfs_ms += ev[1].elapsed_time(ev[2])
        edges += args.pr_iters * E + reach
    t_end.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = st.launch_count - launches0
    ms = t_start.elapsed_time(t_end)
    ms_max, edges_all = reduce_max_sum(ws, ms, edges)
    value = edges_all / (ms_max / 1e3) / 1e9

    # roofline of the PageRank iteration kernel (pr_flat_step + its fix-up
    # over the flat live in-edges): one iteration = the difference between a
    # 2k- and a k-iteration call on the same stream (the per-call flattening
    # cancels), after the timed region
    # algorithmic bytes per iteration as the survey of the path defines them
    # (ids, FP64 contribution gather, deletion bits, fragment descriptors,
    # rank/contribution read+write and degree), and the flat kernel's own
    # model (ids + gather per edge, row start/out-degree/write per row)
    pr_bytes = (ins["live_edges"] * (4 + 8) + ins["slots"] / 8 + ins["fragments"] * 12
                + V * (8 + 8 + 4))
    R = int(np.count_nonzero(sn.in_degrees()))
    flat_bytes = ins["live_edges"] * (4 + 8) + R * (4 + 4 + 8)
    k = args.pr_iters
    diffs = []
    for _ in range(3):
        _, t1 = _timed(stream, lambda: sn.pagerank_pull(k, 0.85, out=pr_dev))
        _, t2 = _timed(stream, lambda: sn.pagerank_pull(2 * k, 0.85, out=pr_dev))
        diffs.append((t2 - t1) / k)
    launch_s = statistics.median(diffs) / 1e3
    peak, peak_kind = measured_peak()
    achieved = pr_bytes / launch_s / 1e9
    # the committed ncu figure is for the default workload only
    traffic = profiled_traffic() if (args.scale, args.levels) == (24, 8) else None
    roofline = {"bound": "hbm", "kernel": "pr_flat_step", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                               if peak_kind == "measured" else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": pr_bytes,
                "bytes_model": "E_live*(4+8) + slots/8 + fragments*12 + V*(8+8+4)",
                "flat_bytes_per_launch": flat_bytes,
                "flat_bytes_model": "12 B per live in-edge (4 B id + 8 B gathered "
                                    "contribution) + 16 B per vertex with in-edges",
                "frac_flat_model": flat_bytes / launch_s / 1e9 / peak,
                "launch_ms": launch_s * 1e3,
                "launch_ms_source": "CUDA events on the store's stream: "
                                    "(t(2k iterations) - t(k iterations)) / k, median of 3",
                "pr_call_ms": pr_ms / args.steps,
                "traffic": traffic["dram_bytes_per_launch_scaled"] if traffic else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one "
                                  "full-size launch (profiles/pr_flat_step_rmat24.md)"
                                  if traffic else None}

    # BFS of the step, against the per-root byte model of the path's survey:
    # sum over roots of (4 B id + 4 B neighbour level per reached out-edge)
    # + 4 B level per vertex; the 12 B per reached fragment term is left out,
    # so the figure is a lower bound of that model. The multi-source and
    # bottom-up steps read fewer bytes than the model charges, so this is the
    # effective bandwidth of the BFS phase (all its kernels), not a DRAM count.
    bfs_s = bfs_ms / args.steps / 1e3
    bfs_bytes = 8 * reach + 4 * V * len(roots)
    bfs_roofline = {"bound": "hbm", "kernels": "BFS phase of the step (%s-source)"
                    % ("multi" if args.bfs == "multi" else "single"),
                    "achieved": bfs_bytes / bfs_s / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": bfs_bytes / bfs_s / 1e9 / peak,
                    "algorithmic_bytes_per_step": bfs_bytes,
                    "bytes_model": "sum over roots of 8*E_reach + 4*V (fragment term "
                                   "omitted: lower bound)",
                    "ms_per_step": bfs_s * 1e3, "roots": len(roots),
                    "note": "effective bandwidth: with --bfs multi the roots share one "
                            "bit-parallel traversal, so the per-root model charges bytes the "
                            "kernels never read and frac can exceed 1; --bfs single gives "
                            "the one-root kernels' figure"}

    # e2e: newest level re-ingested from host, snapshot reopened, results to host
    e2e = None
    if not args.no_e2e:
        sn.close()
        sn = None
        e2e = run_e2e(args, ws, st, hg, V, E, roots, stream)

    ext = None
    if not args.no_extras:
        ext = extras(args, st, stream, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(hg, spec, roots, args)

    line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": ws,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded R-MAT generator, no dataset)",
            "config": dict(cfg, l2="inputs larger than L2: store %.1f GB on the device"
                           % (st.device_bytes / 1e9)),
            "kernels": {"flatten_in_csr": {"ms_per_step": flat_ms / args.steps},
                        "pagerank_pull": {"ms_per_step": pr_ms / args.steps,
                                          "includes": "the in-CSR flatten",
                                          "gteps": args.pr_iters * E * args.steps / (pr_ms / 1e3) / 1e9},
                        "bfs": {"ms_per_step": bfs_ms / args.steps,
                                "gteps": (edges - args.pr_iters * E * args.steps)
                                / (bfs_ms / 1e3) / 1e9, "last_reach_edges": reach}},
            "graph": {"max_nodes": V, "live_edges": E, "in_slots": ins["slots"],
                      "in_fragments": ins["fragments"], "levels": hg.num_levels,
                      "host_build_s": build_s, "ingest_s": ingest_s},
            "roofline": roofline, "bfs_roofline": bfs_roofline, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "cpu_baseline": cpu, "extras": ext}
    if rank == 0:
        emit(line, args)
    if sn is not None:
        sn.close()
    st.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_e2e(args, ws, st, hg, V, E, roots, stream):
    """The step through the C ABI with host buffers: every step replaces the
    newest level (dropped, then rebuilt on the device from its edge delta in
    pinned host memory with lg_store_build_level), opens the snapshot,
    flattens its in-CSR, and copies the ranks and BFS levels to pinned host
    memory.  The same with the host-built level ingested through
    lg_store_ingest_level is reported as host_level.  Then one more step with
    a synchronisation after each phase (no overlap) gives the breakdown."""
    import torch
    # two sets of host result buffers: a pipelined step writes the set its
    # predecessor is not still receiving
    pr_bufs = [torch.empty(V, dtype=torch.float64).pin_memory() for _ in range(2)]
    lv_bufs = [torch.empty((len(roots), V), dtype=torch.int32).pin_memory() for _ in range(2)]
    cur = [0]
    L = hg.num_levels - 1
    desc = hg.level_desc(L)
    src, dst, dsrc, ddst, w = hg.level_input(L)

    def pin(a):
        return None if a is None else torch.from_numpy(a.view(np.int32)).pin_memory()
    p_src, p_dst, p_dsrc, p_ddst, p_w = (pin(x) for x in (src, dst, dsrc, ddst, w))

    def load(kind):
        st.drop_level()
        if kind == "device":
            st.build_level(V, p_src, p_dst, p_w, p_dsrc, p_ddst)
        else:
            st.ingest_level(desc)

    def bfs():
        lv_host = lv_bufs[cur[0]]
        if args.bfs == "multi":
            _, rs = s2.bfs_multi(roots, out=lv_host)
            return sum(r.reach_edges for r in rs)
        reach = 0
        for i, r in enumerate(roots):
            _, res = s2.bfs(int(r), out=lv_host[i])
            reach += res.reach_edges
        return reach

    s2 = None

    def analytics(phase=None, overlap=True, pipeline=False):
        # overlap: the BFS levels (16 x 4 B per vertex) go to the host on the
        # store's copy stream (LG_OUTPUT_ASYNC) while PageRank runs.
        # pipeline: in addition the step does not wait for its copies; the
        # ranks reach the host while the next step rebuilds its level
        nonlocal s2
        pr_host = pr_bufs[cur[0]]
        s2 = st.snapshot()
        if phase:
            phase("snapshot_open")
        s2.flatten(1)
        if overlap:
            if not pipeline:
                st.set_output_mode("async")
            reach = bfs()
            if phase:
                phase("bfs")
            s2.pagerank_pull(args.pr_iters, 0.85, out=pr_host)
            if not pipeline:
                st.sync()                    # every result of the step is on the host
                st.set_output_mode("sync")
            if phase:
                phase("pagerank_and_copies_to_host")
        else:
            s2.pagerank_pull(args.pr_iters, 0.85, out=pr_host)
            if phase:
                phase("flatten_pagerank_to_host")
            reach = bfs()
            if phase:
                phase("bfs_to_host")
        s2.close()
        if pipeline:
            cur[0] ^= 1
        return reach

    def measure(kind, overlap=True, pipeline=False):
        load(kind)
        analytics(overlap=overlap)
        st.sync()
        barrier(ws)
        h0, d0 = st.transfer_bytes()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        edges = 0
        if pipeline:
            st.set_output_mode("async")
        e0.record(stream)
        for _ in range(args.steps):
            load(kind)
            edges += args.pr_iters * E + analytics(overlap=overlap, pipeline=pipeline)
        st.sync()                            # the last step's results are on the host
        if pipeline:
            st.set_output_mode("sync")
        e1.record(stream)
        stream.synchronize()
        h1, d1 = st.transfer_bytes()
        ms = e0.elapsed_time(e1)
        ms_max, edges_all = reduce_max_sum(ws, ms, edges)
        return {"value": edges_all / (ms_max / 1e3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": (h1 - h0) // args.steps,
                "d2h_bytes_per_step": (d1 - d0) // args.steps,
                "ms_per_step": ms_max / args.steps}

    out = measure("device", pipeline=True)
    out["includes"] = ("newest level rebuilt on the device from its edge delta (pinned host "
                       "arrays) + snapshot open + in-CSR flatten + BFS + PageRank, results "
                       "copied to pinned host memory on the store's copy stream (BFS levels "
                       "while PageRank runs, the ranks while the next step rebuilds its "
                       "level, into alternating host buffers); every copy of every step "
                       "inside the timed region")
    stepwise = measure("device")
    stepwise["includes"] = ("as the main figure, every step waiting for its own results "
                            "before the next one starts")
    out["step_synchronous"] = stepwise
    host = measure("host")
    host["includes"] = "as above, the level built on the host and ingested"
    out["host_level"] = host
    sync = measure("device", overlap=False)
    sync["includes"] = "as the main figure, every result copied back before the next call"
    out["sync_output"] = sync
    # phase breakdown of one more device-built step (host clock, synchronised)
    phases = {}
    t = [time.perf_counter()]

    def phase(name):
        st.sync()
        now = time.perf_counter()
        phases[name] = (now - t[0]) * 1e3
        t[0] = now
    st.drop_level()
    st.sync()
    t[0] = time.perf_counter()
    st.build_level(V, p_src, p_dst, p_w, p_dsrc, p_ddst)
    phase("build_level")
    analytics(phase, overlap=False)
    out["phases_ms"] = phases
    return out


def _timed(stream, fn):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r = fn()
    e1.record(stream)
    stream.synchronize()
    return r, e0.elapsed_time(e1)


def extras(args, st, stream, device):
    """Secondary kernels, each timed once with CUDA events on the store's
    stream after a warm-up call: SSSP / triangle counting / SCC on the main
    store; batched vs plain BC and the PPR block on a symmetric Kronecker
    store; adjoint vs forward PageRank on a weighted R-MAT."""
    import torch
    import numpy as np
    from llama_b200 import HostGraph, Store, workloads
    from llama_b200.graph import ppr
    out = {}
    dev = f"cuda:{device}"

    def guard(name, fn):
        try:
            out[name] = fn()
        except Exception as e:      # a failing extra is reported, not fatal
            out[name] = {"error": str(e)[:300]}

    def on_main():
        sn = st.snapshot()
        try:
            V, E = sn.max_nodes, sn.num_edges
            res = {}
            roots = workloads.pick_roots(sn.out_degrees(), 8, seed=13)
            dist = torch.empty(V, dtype=torch.int32, device=dev)
            sn.sssp(int(roots[0]), 32, out=dist)
            reach, ms, rounds, buckets, relax = 0, 0.0, 0, 0, 0
            for r in roots:
                (_, rr), t = _timed(stream, lambda: sn.sssp(int(r), 32, out=dist))
                reach += rr.reach_edges
                ms += t
                rounds += rr.rounds
                buckets += rr.buckets
                relax += rr.relaxations
            res["sssp_delta32_8roots"] = {"ms": ms, "gteps": reach / (ms / 1e3) / 1e9,
                                          "rounds": rounds, "buckets": buckets,
                                          "relaxations_per_reached_edge": relax / max(reach, 1)}
            # the same roots on the snapshot with its out-CSR flattened once
            _, fms = _timed(stream, lambda: sn.flatten(0))
            reach, ms = 0, 0.0
            for r in roots:
                (_, rr), t = _timed(stream, lambda: sn.sssp(int(r), 32, out=dist))
                reach += rr.reach_edges
                ms += t
            sn.unflatten()
            res["sssp_delta32_8roots_flat"] = {"ms": ms, "gteps": reach / (ms / 1e3) / 1e9,
                                               "flatten_out_csr_ms": fms,
                                               "includes": "not the one flatten"}
            sn.triangle_count()
            tc, ms = _timed(stream, sn.triangle_count)
            res["triangle_count"] = {"ms": ms, "triangles": tc.triangles,
                                     "gteps": E / (ms / 1e3) / 1e9}
            age = torch.randint(0, 80, (V,), dtype=torch.int32, device=dev,
                                generator=torch.Generator(device=dev).manual_seed(16))
            tcnt = torch.empty(V, dtype=torch.int32, device=dev)
            sn.avg_teen_cnt(age, 0, out=tcnt)
            (_, trr), ms = _timed(stream, lambda: sn.avg_teen_cnt(age, 0, out=tcnt))
            res["avg_teen_cnt"] = {"ms": ms, "average": trr.average,
                                   "gteps": E / (ms / 1e3) / 1e9,
                                   "includes": "in-CSR flatten for the call"}
            lab = torch.empty(V, dtype=torch.int64, device=dev)
            sn.scc(out=lab)
            (_, sr), ms = _timed(stream, lambda: sn.scc(out=lab))
            res["scc"] = {"ms": ms, "components": sr.components, "gteps": E / (ms / 1e3) / 1e9}
            return res
        finally:
            sn.close()

    def on_kron():
        spec = workloads.kronecker_symmetric(scale=args.kron_scale, seed=6, levels=4)
        hg = HostGraph.from_spec(spec)
        with Store(device=device, stream=stream.cuda_stream) as s2:
            s2.ingest(hg)
            snaps = [s2.snapshot(l) for l in range(4)]
            try:
                sn = snaps[-1]
                V, E = sn.max_nodes, sn.num_edges
                src = workloads.pick_roots(sn.out_degrees(), args.bc_sources, seed=14)
                bc = torch.empty(V, dtype=torch.float64, device=dev)
                sn.bc(src[:64], batched=True, out=bc)
                tb = statistics.median(
                    _timed(stream, lambda: sn.bc(src, batched=True, out=bc))[1] for _ in range(3))
                # the speed-up on the same 64 sources, one batch against one by one
                s64 = src[:64]
                t64 = statistics.median(
                    _timed(stream, lambda: sn.bc(s64, batched=True, out=bc))[1] for _ in range(3))
                sn.bc(s64[:2], batched=False, out=bc)
                tp = statistics.median(
                    _timed(stream, lambda: sn.bc(s64, batched=False, out=bc))[1] for _ in range(3))
                res = {"bc": {"graph": f"Kronecker scale {args.kron_scale}, symmetric, 4 levels",
                              "batched_ms_per_source": tb / len(src),
                              "batched_gteps": 2 * E * len(src) / (tb / 1e3) / 1e9,
                              "sources_batched": len(src),
                              "same_64_sources": {"batched_ms": t64, "plain_ms": tp,
                                                  "batched_speedup": tp / t64},
                              "timing": "median of 3 runs each"}}
                seeds = workloads.pick_roots(sn.out_degrees(), 256, seed=15)
                out_ppr = torch.empty((4, V, 256), dtype=torch.float64, device=dev)
                ppr(snaps, seeds[:32], iterations=2, out=out_ppr[:, :, :32].contiguous())
                _, tq = _timed(stream, lambda: ppr(snaps, seeds, iterations=20, out=out_ppr))
                e_all = sum(s.num_edges for s in snaps)
                res["ppr"] = {"K": 256, "iterations": 20, "snapshots": 4, "ms": tq,
                              "gteps": 20 * e_all * 256 / (tq / 1e3) / 1e9}
                return res
            finally:
                for s in snaps:
                    s.close()

    def on_adjoint():
        spec = workloads.rmat_multiversion(scale=args.adjoint_scale, seed=4, levels=1, level0=1.0)
        hg = HostGraph.from_spec(spec)
        with Store(device=device, stream=stream.cuda_stream) as s3:
            s3.ingest(hg)
            with s3.snapshot() as sn:
                V = sn.max_nodes
                off, nb = sn.adjacency(0)
                rng = np.random.default_rng(4)
                raw = rng.uniform(0.5, 1.5, len(nb))
                srcv = np.repeat(np.arange(V), np.diff(off.astype(np.int64)))
                w = torch.tensor(raw / np.bincount(srcv, raw, V)[srcv], device=dev)
                v = rng.exponential(1.0, V)
                v = torch.tensor(v / v.sum(), device=dev)
                u = torch.empty(V, dtype=torch.float64, device=dev)
                sn.pagerank_fwd(w, torch.full((V,), 1.0 / V, dtype=torch.float64, device=dev),
                                0.85, keep_tape=False, out=u)
                x = torch.empty(V, dtype=torch.float64, device=dev)
                (_, tape, fr), tf = _timed(stream, lambda: sn.pagerank_fwd(w, v, 0.85, out=x))
                # L = sum over 1024 targets of (x_v - 1.2 u_v)^2, u = uniform-teleport scores
                T = torch.tensor(rng.choice(V, 1024, replace=False), device=dev)
                g = torch.zeros(V, dtype=torch.float64, device=dev)
                g[T] = 2 * (x[T] - 1.2 * u[T])
                dw = torch.empty(len(nb), dtype=torch.float64, device=dev)
                dv = torch.empty(V, dtype=torch.float64, device=dev)
                (_, _, br), tb = _timed(stream, lambda: tape.backward(g, dw, dv))
                tape.close()
                return {"graph": f"R-MAT scale {args.adjoint_scale}, FP64 weights U[0.5,1.5] "
                                 "row-normalised, Dirichlet(1) teleport, tol 1e-12",
                        "forward_ms": tf, "forward_iterations": fr.iterations,
                        "backward_ms": tb, "backward_iterations": br.iterations,
                        "backward_over_forward": tb / tf}

    guard("kronecker", on_kron)
    guard("main_store", on_main)
    guard("adjoint", on_adjoint)
    return out


def cpu_baseline(hg, spec, roots, args):
    """Reference OpenMP kernels on this host's cores, one step (bounded)."""
    from oracle.bind import Reference, ref_available
    if not ref_available():
        return None
    t0 = time.time()
    R = Reference(spec.max_nodes)
    for l in range(hg.num_levels):
        R.add_level(*hg.level_input(l)[:4])
    build_s = time.time() - t0
    deg = R.degrees(-1)
    E = int(deg.sum())
    _, t_pr = R.pagerank_pull(-1, args.pr_iters, 0.85)
    t_bfs, reach = 0.0, 0
    for r in roots:
        lv, t = R.bfs(-1, int(r))
        t_bfs += t
        reach += int(deg[lv < 2147483646].sum(dtype=np.int64))
    gteps = (args.pr_iters * E + reach) / (t_pr + t_bfs) / 1e9
    return {"value": gteps, "unit": "GTEPS", "cores": Reference.max_threads(),
            "kind": "reference",
            "sample": f"one full step (pagerank_double x{args.pr_iters} + sssp_unweighted "
                      f"BFS from {len(roots)} roots) on the same store, run() time only",
            "pagerank_s": t_pr, "bfs_s": t_bfs, "store_build_s": build_s}


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max_sum(ws, ms, edges):
    """(max over ranks of ms, sum over ranks of edges): the job's time is its
    slowest rank's, its work all ranks' work."""
    if ws == 1:
        return ms, edges
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    e = torch.tensor([float(edges)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_lg(args)


if __name__ == "__main__":
    main()
