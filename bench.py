"""Benchmark of the B200 compute path on synthetic R-MAT graphs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  Workload: the directed R-MAT scale-22 graph
(4,194,304 nodes, edge factor 16, a/b/c/d = .57/.19/.19/.05, seed 1,
self-loops and repeats dropped, ids relabelled by sorted random int64
external ids).  A step is one batch of the hot path over that graph:

- batched: 1,024 BFS searches from seeded random sources with per-source
  depth caps U{1..16}, as one bit-packed boolean SpMM (wc_bfs_batched);
- plain: the same searches one wc_bfs call each (a sample of them per step,
  scaled by edges traversed);
- PageRank: FP64, damping 0.85, tol 1e-10 (stop at delta < live × tol),
  at most 100 iterations (wc_pagerank).

`value` is the batched aggregate GTEPS (Σ over sources of the edges a
push-only BFS from that source traverses, the reference's edges_traversed,
÷ time) over all ranks; the plain path and PageRank are reported beside it.
Inputs are device-resident when the timed region starts (`value`); `e2e`
times the same work through the C ABI from host buffers, copies included.
The graph (≈1.6 GB of CSR + CSC on the device) is larger than L2 and L2 is
also flushed between timed steps.  Multi-GPU runs shard the sources across
ranks (weak scaling, no exchange).  The CPU baseline is the C++ oracle
(warren-core's kernels restated) on a bounded sample on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE = int(os.environ.get("WARREN_BENCH_SCALE", "22"))
WIDTH = 1024
PLAIN_SAMPLE = 32  # plain-path searches timed per step
SEED = 1


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_graph():
    import pg_warren_b200 as W
    g = W.rmat(SCALE, 16, 0.57, 0.19, 0.19, SEED)
    return g


def sources_and_caps(n, count=WIDTH, seed=SEED):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, count).astype(np.uint64), rng.integers(1, 17, count).astype(np.uint32)


def push_edges(offsets, depth, caps=None):
    """Edges a push-only BFS traverses: Σ out-degree over expanded nodes
    (those reached at a depth below the cap)."""
    deg = np.diff(offsets).astype(np.int64)
    return deg, None


def oracle_edges(og, sources, caps):
    import oracle as O
    _, e = O.bfs_depths(og, sources, caps)
    return e


# --------------------------------------------------------------- reference arm

def reference_arm(args):
    """warren-core's CPU kernels (the C++ restatement; the Rust crate cannot
    be built here) on all host threads, on bounded samples of the same
    workload: each step = BFS searches from a sample of the sources."""
    import oracle as O
    O.build()
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    g = make_graph()
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, reverse=False)
    src, caps = sources_and_caps(g.id_space)
    cores = O.lib().wo_threads()
    sample = max(cores, 8)
    for _ in range(args.warmup):
        O.bfs_depths(og, src[:2], caps[:2])
    times, edges = [], []
    for step in range(args.steps):
        sl = slice((step * sample) % WIDTH, (step * sample) % WIDTH + sample)
        t0 = time.perf_counter()
        _, e = O.bfs_depths(og, src[sl], caps[sl])
        times.append(time.perf_counter() - t0)
        edges.append(int(e.sum()))
    gteps = sum(edges) / sum(times) / 1e9
    line = {
        "metric": "BFS GTEPS & PageRank iters/s, batched vs plain on 1 B200, % HBM roofline",
        "impl": "reference", "value": gteps, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"rmat{SCALE}-bfs-{WIDTH}-sources-caps-1..16",
                   "scale": SCALE, "edge_factor": 16, "sources": WIDTH},
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": cores, "kind": "port",
                         "sample": f"{sample} of the {WIDTH} BFS searches per step"},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# --------------------------------------------------------------- GPU arm

def flush_l2(torch, buf):
    buf.add_(1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="warren")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import pg_warren_b200 as W
    from pg_warren_b200 import _abi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    peak, peak_kind = measured_peaks()

    t0 = time.time()
    g = make_graph()
    n, m = g.id_space, g.edges
    gv = g.upload()
    setup_s = time.time() - t0
    src_all, caps_all = sources_and_caps(n)
    # Weak scaling: each rank takes its own 1,024 sources.
    src_all, caps_all = sources_and_caps(n, WIDTH, SEED + rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        ms = []
        for _ in range(steps):
            flush_l2(torch, flush)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        barrier()
        return ms

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    launches = {"count": 0}
    result = {}

    # ---- plain path: one wc_bfs per source (device outputs)
    depth_d = torch.empty(n, dtype=torch.int32, device=dev)
    via_d = torch.empty(n, dtype=torch.int64, device=dev)
    plain_edges = []

    def plain_step():
        e = 0
        for s, c in zip(src_all[:PLAIN_SAMPLE], caps_all[:PLAIN_SAMPLE]):
            _, _, st = W.bfs_depths(gv, [int(s)], max_depth=int(c), depth_out=depth_d,
                                    via_out=via_d)
            e += st.edges_traversed
        plain_edges.append(e)

    ms_plain = timed(plain_step, max(1, args.steps // 2), 1)
    plain_gteps = plain_edges[-1] / (statistics.median(ms_plain) * 1e-3) / 1e9
    result["plain_bfs_gteps"] = plain_gteps

    # ---- PageRank
    ranks_d = torch.empty(n, dtype=torch.float64, device=dev)
    pr_iters = []

    def pr_step():
        r = W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100), out=ranks_d, stream=stream)
        pr_iters.append(r.iterations)

    with Clocks(local) as clocks:
        ms_pr = timed(pr_step, args.steps, args.warmup)
    it = pr_iters[-1]
    pr_ms = statistics.median(ms_pr)
    pr_iters_s = it / (pr_ms * 1e-3)
    pr_bytes_iter = 4 * (n + 1) + 4 * m + 24 * n
    result["pagerank"] = {"iterations": it, "ms": pr_ms, "iters_per_s": pr_iters_s,
                          "gbs": pr_bytes_iter * it / (pr_ms * 1e-3) / 1e9,
                          "margin": W.api.last_margin(gv)}

    # ---- batched path
    batched = None
    try:
        depth_b = torch.empty((WIDTH, n), dtype=torch.uint8, device=dev)
        edges_b = torch.empty(WIDTH, dtype=torch.int64, device=dev)
        sched = W.autotune(gv, "bfs", WIDTH)
        result["schedule"] = {"columns_per_pass": sched.columns_per_pass,
                              "blocks_per_sm": sched.blocks_per_sm}

        def batched_step():
            W.bfs_batched(gv, src_all, caps_all, depth_out=depth_b, edges_out=edges_b)

        with Clocks(local) as clocks_b:
            ms_b = timed(batched_step, args.steps, args.warmup)
        total_edges = int(edges_b.sum().item())
        b_ms = statistics.median(ms_b)
        batched_gteps = total_edges / (b_ms * 1e-3) / 1e9
        levels = int(depth_b[depth_b != 255].max().item())
        b_bytes_level = 4 * (n + 1) + 4 * m + n * WIDTH // 4
        result["batched"] = {"ms": b_ms, "gteps": batched_gteps, "levels": levels,
                             "edges": total_edges,
                             "gbs_dense_operand_bound": levels * b_bytes_level / (b_ms * 1e-3) / 1e9}
        batched = True
    except W.api.Unsupported:
        batched = False

    line = {
        "metric": "BFS GTEPS & PageRank iters/s, batched vs plain on 1 B200, % HBM roofline",
        "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": f"rmat{SCALE}-bfs-{WIDTH}-sources-caps-1..16+pagerank-f64",
                   "scale": SCALE, "nodes": n, "edges": m, "edge_factor": 16,
                   "sources_per_rank": WIDTH, "l2": "inputs larger than L2; flushed between steps"},
    }
    if not batched:
        # Headline falls back to the plain path until the batched kernel lands.
        line["value"] = plain_gteps * world
        line["ms_per_step"] = statistics.median(ms_plain)
    else:
        ms_max = max_over_ranks(result["batched"]["ms"])
        line["value"] = world * result["batched"]["edges"] / (ms_max * 1e-3) / 1e9
        line["ms_per_step"] = ms_max
        line["batched"] = result["batched"]
        line["batched_vs_plain"] = result["batched"]["gteps"] / plain_gteps
        line["schedule"] = result["schedule"]
        clocks = clocks_b
    line["plain_bfs_gteps"] = plain_gteps
    line["pagerank_iters_per_s"] = pr_iters_s
    line["pagerank"] = result["pagerank"]
    achieved = result["pagerank"]["gbs"]
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": None,
                        "kernel": "pr_iter_kernel (PageRank iteration)",
                        "peak_kind": peak_kind}
    line["clocks"] = clocks.summary()
    line["setup_s"] = setup_s
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
