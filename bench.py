"""Benchmark of the B200 compute path on synthetic R-MAT graphs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).

Workload (the batched-traversal configuration): the directed R-MAT scale-22
graph (4,194,304 nodes, edge factor 16, a/b/c/d = .57/.19/.19/.05, seed 1;
self-loops and repeats dropped, ids relabelled by sorted random int64
external ids; 65,241,322 stored edges) and 1,024 seeded random sources with
per-source depth caps drawn from U{1..16}.  A step is one batched BFS of
the 1,024 sources: one bit-packed boolean SpMM per level in a persistent
kernel, each pass of sources replayed from a captured CUDA graph
(wc_bfs_batched).

- value: aggregate GTEPS over all ranks = Σ over sources of edges_traversed
  (the out-degree summed over the nodes a push-only BFS from the source
  expands, as warren-core counts it) ÷ device time (CUDA events on the
  call's stream, inputs resident in HBM, max over ranks).
- e2e: the same metric through the public call with host buffers: sources
  and caps copied from pinned host memory, the 1,024 × n depth matrix and
  the edge counts copied back to pinned host memory, inside the timed step.
- roofline: msbfs_level_kernel (one level of a pass = one boolean SpMM
  iteration over k columns); algorithmic bytes per level 4(n+1) + 4m +
  n·k·(1/8 + 1/8) (CSC offsets and targets once, the frontier operand read
  and written once), timed by CUDA events the library records around the
  level launches on the call's stream during the timed steps.
- Beside it: the plain per-source GPU BFS (wc_bfs, a sample of the sources),
  FP64 PageRank (damping 0.85, tol 1e-10 × live nodes, at most 100
  iterations) in iterations/s with its own roofline, and the CPU baseline:
  the oracle (warren-core's kernels restated in C++) on the host cores, on a
  bounded sample of the sources.

Inputs are larger than L2 (CSC 0.28 GB, frontier snapshots ≈ 4.5 GB), and a
256 MiB buffer is also written between timed steps.  Multi-GPU runs give
each rank its own 1,024 sources on a replica of the graph: weak scaling, no
exchange on the data path.
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

METRIC = "BFS GTEPS & PageRank iters/s, batched vs plain on 1 B200, % HBM roofline"
SCALE = 22
WIDTH = 1024
PLAIN_SAMPLE = 32
SEED = 1
CPU_BUDGET_S = 12.0
# DRAM bytes per algorithmic byte of a pull level, from the ncu capture of
# msbfs_level_kernel on the same workload at R-MAT 20 (the full-size launch
# is past the capture-size rule): traffic scales with the level's units.
LEVEL_TRAFFIC_RATIO = (256.51 + 113.99) / 337.0
LEVEL_TRAFFIC_SOURCE = ("dram__bytes_read.sum + dram__bytes_write.sum of one pull level at "
                        "R-MAT 20 (profiles/msbfs_level_kernel_rmat20_1024src.md), scaled "
                        "by the algorithmic bytes")


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        if "hbm_gbs" in p:
            return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            time.sleep(0.3)
        except OSError:
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
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_graph():
    import pg_warren_b200 as W
    return W.rmat(SCALE, 16, 0.57, 0.19, 0.19, SEED)


def sources_and_caps(n, rank=0):
    rng = np.random.default_rng(SEED + 1000 * rank)
    return rng.integers(0, n, WIDTH).astype(np.uint64), rng.integers(1, 17, WIDTH).astype(np.uint32)


def config(n, m, **extra):
    c = {"workload": f"rmat{SCALE}-batched-bfs-{WIDTH}-sources-caps-U1..16",
         "scale": SCALE, "edge_factor": 16, "nodes": n, "edges": m, "sources_per_rank": WIDTH,
         "l2": "inputs larger than L2; 256 MiB buffer written between timed steps"}
    c.update(extra)
    return c


def cpu_bfs(offsets, targets, sources, caps, budget_s, check=None, batched=True):
    """The oracle (warren-core's traversal restated in C++) on all host
    threads, over as many of the sources as fit the budget: (GTEPS, sources
    run, threads, seconds).  `batched`: the reference's own batched shape
    (compute/centrality/multi_source.rs: 64 sources a word, parallel over
    the frontier); otherwise one LevelSearch per source, the searches in
    parallel.  `check(slice, depths, edges)`, if given, is called outside
    the timed region with each batch's results, to compare them with the
    GPU's."""
    import oracle as O
    O.build()
    og = O.Graph.from_csr(len(offsets) - 1, offsets, targets, reverse=False)
    threads = int(O.lib().wo_threads())
    search = O.bfs_depths_batched64 if batched else O.bfs_depths
    search(og, sources[:1], caps[:1])  # warm
    batch = 64 if batched else max(1, threads)
    done, edges, secs = 0, 0, 0.0
    while done < len(sources) and secs < budget_s:
        sl = slice(done, min(len(sources), done + batch))
        t0 = time.perf_counter()
        d, e = search(og, sources[sl], caps[sl])
        secs += time.perf_counter() - t0
        edges += int(e.sum())
        done = sl.stop
        if check is not None:
            check(sl, d, e)
    return edges / secs / 1e9, done, threads, secs


# --------------------------------------------------------------- reference arm

def reference_arm(args):
    """warren-core's CPU path (restated in C++; the Rust crate has no
    toolchain here) on all host threads; each step a bounded sample of the
    same 1,024 searches.  Rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import oracle as O
    O.build()
    # The graph from the oracle's own copy of the generator: this arm maps
    # no library of the GPU path.
    g = O.rmat(SCALE, 16, 0.57, 0.19, 0.19, SEED)
    src, caps = sources_and_caps(g.id_space)
    per_step = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, reverse=False)
    threads = int(O.lib().wo_threads())
    # The reference's own batched shape (multi_source.rs: 64 sources a word,
    # the frontier's nodes in parallel tasks), the faster of its CPU paths.
    batch = 64
    pos = 0

    def step():
        nonlocal pos
        edges, secs = 0, 0.0
        while secs < per_step:
            idx = [(pos + q) % WIDTH for q in range(batch)]
            pos = (pos + batch) % WIDTH
            t0 = time.perf_counter()
            _, e = O.bfs_depths_batched64(og, src[idx], caps[idx])
            secs += time.perf_counter() - t0
            edges += int(e.sum())
        return edges, secs

    for _ in range(args.warmup):
        step()
    tot_e, tot_s = 0, 0.0
    for _ in range(args.steps):
        e, s = step()
        tot_e += e
        tot_s += s
    gteps = tot_e / tot_s / 1e9
    sample = (f"searches from the {WIDTH} sources, {batch} at a time (one 64-source word), "
              f"≈{per_step:.0f} s per step")
    print(json.dumps({
        "metric": METRIC, "impl": "reference", "value": gteps, "unit": "GTEPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config(g.id_space, g.edges),
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# --------------------------------------------------------------- GPU arm

def executed_levels(depth, caps, columns):
    """Per pass of `columns` sources: the levels whose frontier was
    non-empty (level L runs when some source with cap > L reached a node at
    depth L)."""
    import torch
    k = depth.shape[0]
    total = 0
    for s0 in range(0, k, columns):
        d = depth[s0:s0 + columns]
        reached = torch.where(d == 255, torch.zeros_like(d), d).amax(dim=1).to(torch.int64)
        c = torch.as_tensor(caps[s0:s0 + columns].astype(np.int64), device=d.device)
        last = torch.minimum(reached, c - 1)
        total += int(last.max().item()) + 1
    return total


# --------------------------------------------------------------- the suite
# `python bench.py --suite c1,c2,c3,c4,c5` measures every configuration of
# the path (one JSON object, legs by name); the default run above is the
# batched-traversal line alone.

def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def leg_c1(W, O, torch, dev, stream, peak):
    """R-MAT 16: 64 separate BFS (depth cap 8) and FP64 PageRank (tol
    1e-10), on the GPU and on the oracle, compared."""
    g = W.rmat(16)
    n, m = g.id_space, g.edges
    gv = g.upload()
    og = O.Graph.from_csr(n, g.offsets, g.targets)
    rng = np.random.default_rng(SEED)
    seeds = rng.integers(0, n, 64).astype(np.uint64)
    caps = np.full(64, 8, np.uint32)
    O.bfs_depths(og, seeds, caps)
    t0 = time.perf_counter()
    depth, edges = O.bfs_depths(og, seeds, caps)
    cpu_bfs_s = time.perf_counter() - t0
    dd = torch.empty(n, dtype=torch.int32, device=dev)
    vv = torch.empty(n, dtype=torch.int64, device=dev)
    gpu_edges = 0
    t0 = time.perf_counter()
    for s in seeds:
        _, _, st = W.bfs_depths(gv, [int(s)], max_depth=8, depth_out=dd, via_out=vv)
        gpu_edges += st.edges_traversed
    torch.cuda.synchronize(dev)
    gpu_bfs_s = time.perf_counter() - t0
    exact = True
    for q, s in enumerate(seeds):
        W.bfs_depths(gv, [int(s)], max_depth=8, depth_out=dd, via_out=vv)
        d = dd.cpu().numpy()
        mine = np.where(d == -1, 255, d).astype(np.int64)
        exact &= bool(np.array_equal(mine, depth[q].astype(np.int64)))
    ro, ito = O.pagerank(og, 0.85, 1e-10, 100)[:2]
    t0 = time.perf_counter()
    O.pagerank(og, 0.85, 1e-10, 100)
    cpu_pr_s = time.perf_counter() - t0
    r = W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100))
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        r = W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100))
    gpu_pr_s = (time.perf_counter() - t0) / reps
    return {"graph": {"scale": 16, "nodes": n, "edges": m},
            "bfs": {"searches": 64, "max_depth": 8, "gpu_gteps": gpu_edges / gpu_bfs_s / 1e9,
                    "cpu_gteps": int(edges.sum()) / cpu_bfs_s / 1e9,
                    "cpu_threads": int(O.lib().wo_threads()),
                    "depths_equal_oracle": exact,
                    "edges_equal_oracle": int(edges.sum()) == gpu_edges},
            "pagerank": {"iterations": r.iterations, "oracle_iterations": int(ito),
                         "rel_l1_vs_oracle": float(np.abs(r.values - ro).sum() / ro.sum()),
                         "gpu_ms": gpu_pr_s * 1e3, "cpu_ms": cpu_pr_s * 1e3}}


def _spmv_sweep(W, O, torch, dev, stream, peak, g, cpu):
    n, m = g.id_space, g.edges
    rng = np.random.default_rng(SEED)
    out = {}
    hot = rng.random(n) < 0.01
    wf = 1.0 - rng.random(m)                         # U(0, 1]
    wi = rng.integers(1, 101, m).astype(np.float64)  # U{1..100}
    cases = [("plus_times", wf, 4 * (n + 1) + 12 * m + 16 * n),
             ("min_plus", wi, 4 * (n + 1) + 8 * m + 8 * n),
             ("lor_land", None, 4 * (n + 1) + 4 * m + 2 * n)]
    for sr, w, bytes_it in cases:
        gv = W.GraphVersion(g.offsets, g.targets, w)
        if sr == "plus_times":
            x0 = torch.as_tensor(np.where(hot, 1.0, 0.0), device=dev)
        elif sr == "min_plus":
            x0 = torch.as_tensor(np.where(hot, 0, np.iinfo(np.int64).max).astype(np.int64),
                                 device=dev)
        else:
            x0 = torch.as_tensor(hot.astype(np.uint8), device=dev)
        for transpose in (False, True):
            prod = W.Product(sr, transpose=transpose)
            x = x0.clone()
            y = torch.empty_like(x)
            for _ in range(3):
                W.spmv(gv, prod, x, y, stream=stream.cuda_stream, asynchronous=True)
            torch.cuda.synchronize(dev)
            x = x0.clone()
            a, b = _events(torch)
            a.record(stream)
            for _ in range(20):
                W.spmv(gv, prod, x, y, stream=stream.cuda_stream, asynchronous=True)
                x, y = y, x
            b.record(stream)
            b.synchronize()
            W.load().wc_version_sync(gv.handle, None)
            ms = a.elapsed_time(b) / 20
            gbs = bytes_it / (ms * 1e-3) / 1e9
            out[f"{sr}/{'csc' if transpose else 'csr'}"] = {
                "us_per_iteration": ms * 1e3, "gbs": gbs, "frac": gbs / peak,
                "ge_per_s": m / (ms * 1e-3) / 1e9}
        if cpu:
            og = O.Graph.from_csr(n, g.offsets, g.targets, w)
            xs = x0.cpu().numpy()
            ys = np.empty_like(xs)
            sid = {"plus_times": 0, "min_plus": 1, "lor_land": 5}[sr]
            t0 = time.perf_counter()
            O.product(og, sid, xs, ys, transpose=True)
            sec = time.perf_counter() - t0
            out[f"{sr}/cpu"] = {"ge_per_s": m / sec / 1e9, "threads": int(O.lib().wo_threads()),
                                "sample": "one iteration over the CSC"}
            # Parity at this size: the same product on the device.
            yg = torch.empty_like(x0)
            W.spmv(gv, W.Product(sr, transpose=True), x0.clone(), yg)
            yg = yg.cpu().numpy()
            if sr == "plus_times":
                rel = np.abs(yg - ys) / np.maximum(np.abs(ys), 1e-300)
                out[f"{sr}/parity"] = {"max_rel_vs_oracle": float(rel.max()),
                                       "rows_bit_exact": float(np.mean(yg == ys))}
            else:
                out[f"{sr}/parity"] = {"bit_exact_vs_oracle": bool(np.array_equal(yg, ys))}
        del gv
    return out


def spmv_point(W, torch, dev, stream, peak, g):
    """plus_times f64 over the reverse CSR (pull, the reference's transpose
    product), R-MAT 22, 20 iterations from a 1% vector: spmv_pull_kernel's
    fraction of the roofline, bytes 4(n+1) + 12m + 16n an iteration."""
    n, m = g.id_space, g.edges
    rng = np.random.default_rng(SEED)
    w = 1.0 - rng.random(m)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    x0 = torch.as_tensor(np.where(rng.random(n) < 0.01, 1.0, 0.0), device=dev)
    prod = W.Product("plus_times", transpose=True)
    x, y = x0.clone(), torch.empty_like(x0)
    for _ in range(3):
        W.spmv(gv, prod, x, y, stream=stream.cuda_stream, asynchronous=True)
    torch.cuda.synchronize(dev)
    a, b = _events(torch)
    a.record(stream)
    for _ in range(20):
        W.spmv(gv, prod, x, y, stream=stream.cuda_stream, asynchronous=True)
        x, y = y, x
    b.record(stream)
    b.synchronize()
    W.load().wc_version_sync(gv.handle, None)
    ms = a.elapsed_time(b) / 20
    bytes_it = 4 * (n + 1) + 12 * m + 16 * n
    gbs = bytes_it / (ms * 1e-3) / 1e9
    return {"kernel": "spmv_pull_kernel", "semiring": "plus_times", "dtype": "f64",
            "us_per_iteration": ms * 1e3, "bytes_per_iteration": bytes_it,
            "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}


def leg_c2(W, O, torch, dev, stream, peak):
    """Semiring SpMV sweep: R-MAT 22 and G(n,m) of the same n and m."""
    g = W.rmat(22)
    res = {"rmat22": _spmv_sweep(W, O, torch, dev, stream, peak, g, True)}
    e = W.gnm(g.id_space, g.edges)
    res["gnm"] = _spmv_sweep(W, O, torch, dev, stream, peak, e, False)
    res["graphs"] = {"rmat22": {"nodes": g.id_space, "edges": g.edges},
                     "gnm": {"nodes": e.id_space, "edges": e.edges}}
    return res


def leg_c3(W, O, torch, dev, stream, peak, g=None):
    """Batched min-plus (1,024 sources, int32 weights 1..100, caps U{1..16})
    and 256 personalised PageRank seed sets (sizes log-uniform 1..1000)."""
    g = g if g is not None else W.rmat(22)
    n, m = g.id_space, g.edges
    rng = np.random.default_rng(SEED)
    wi = rng.integers(1, 101, m).astype(np.float64)
    gv = W.GraphVersion(g.offsets, g.targets, wi)
    src = rng.integers(0, n, 1024).astype(np.uint64)
    caps = rng.integers(1, 17, 1024).astype(np.uint32)
    d = torch.empty((1024, n), dtype=torch.int64, device=dev)
    it = torch.empty(1024, dtype=torch.int32, device=dev)
    W.minplus_batched(gv, src, caps, dist_out=d, iterations_out=it)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    W.minplus_batched(gv, src, caps, dist_out=d, iterations_out=it)
    torch.cuda.synchronize(dev)
    mp_s = time.perf_counter() - t0
    iters = int(it.sum().item())
    # Parity at this size: the oracle's sssp_vector loop on 8 sources.
    mp_parity = None
    if O is not None:
        og = O.Graph.from_csr(n, g.offsets, g.targets, wi)
        pick = np.arange(0, 1024, 128)
        do, ito = O.sssp_i64(og, src[pick], caps[pick])
        got = d[torch.as_tensor(pick, device=dev)].cpu().numpy()
        mp_parity = {"checked_sources": int(len(pick)),
                     "bit_exact": bool(np.array_equal(got, do) and np.array_equal(
                         it.cpu().numpy()[pick], ito.astype(np.int32)))}
        del og
    del d
    # The plain per-source path: the sssp_vector loop, one SpMV a step
    # (min_plus over the reverse CSR, accumulate min) on a sample of the
    # sources, until no distance falls or the cap.
    prod = W.Product("min_plus", transpose=True, accumulate="min")
    plain_s, plain_cols, plain_iters = 0.0, 0, 0
    xs = torch.empty(n, dtype=torch.int64, device=dev)
    ys = torch.empty(n, dtype=torch.int64, device=dev)
    for q in range(8):
        xs.fill_(np.iinfo(np.int64).max)
        xs[int(src[q])] = 0
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for step in range(int(caps[q])):
            ys.copy_(xs)
            W.spmv(gv, prod, xs, ys)
            plain_iters += 1
            fell = bool((ys < xs).any().item())
            xs, ys = ys, xs
            if not fell:
                break
        torch.cuda.synchronize(dev)
        plain_s += time.perf_counter() - t0
        plain_cols += 1
    plain_per_source = plain_s / plain_cols
    gu = g.upload()
    sizes = np.exp(rng.uniform(0, np.log(1000), 256)).astype(np.int64)
    sets = [rng.choice(n, int(s), replace=False) for s in sizes]
    psched = W.autotune(gu, "ppr", 256)
    r = torch.empty((256, n), dtype=torch.float64, device=dev)
    pit = torch.empty(256, dtype=torch.int32, device=dev)
    W.ppr_batched(gu, sets, W.PageRank(0.85, 1e-10, 100), ranks_out=r, iterations_out=pit)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    W.ppr_batched(gu, sets, W.PageRank(0.85, 1e-10, 100), ranks_out=r, iterations_out=pit)
    torch.cuda.synchronize(dev)
    ppr_s = time.perf_counter() - t0
    # Parity at this size: the oracle's seeded PageRank on 3 of the sets.
    ppr_parity = None
    if O is not None:
        ogu = O.Graph.from_csr(n, g.offsets, g.targets)
        rels, its_equal = [], True
        for q in (0, 100, 200):
            seed = np.zeros(n)
            seed[sets[q]] = 1.0
            ro, ito, _, _ = O.pagerank(ogu, 0.85, 1e-10, 100, seed=seed)
            rels.append(float(np.abs(r[q].cpu().numpy() - ro).sum() / np.abs(ro).sum()))
            its_equal &= int(pit[q].item()) == ito
        ppr_parity = {"checked_sets": 3, "max_rel_l1_vs_oracle": max(rels),
                      "iterations_equal": bool(its_equal)}
        del ogu
    del r
    seeds = []
    for q in range(8):
        seed = torch.zeros(n, dtype=torch.float64, device=dev)
        seed[torch.as_tensor(sets[q].astype(np.int64), device=dev)] = 1.0
        seeds.append(seed)
    rk = torch.empty(n, dtype=torch.float64, device=dev)
    W.pagerank(gu, None, W.PageRank(0.85, 1e-10, 100, seed=seeds[0]), out=rk)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for seed in seeds:
        W.pagerank(gu, None, W.PageRank(0.85, 1e-10, 100, seed=seed), out=rk)
    torch.cuda.synchronize(dev)
    plain_ppr_s = (time.perf_counter() - t0) / len(seeds)
    return {"minplus": {"sources": 1024, "seconds": mp_s, "column_iterations": iters,
                        "gteps_relaxations": iters * m / mp_s / 1e9,
                        "plain_per_source_ms": plain_per_source * 1e3,
                        "plain_sample": f"{plain_cols} sources, {plain_iters} loop steps",
                        "batched_vs_plain": plain_per_source * 1024 / mp_s,
                        "parity": mp_parity},
            "ppr": {"seed_sets": 256, "seconds": ppr_s, "iterations_max": int(pit.max().item()),
                    "columns_per_pass": psched.columns_per_pass,
                    "per_set_ms": ppr_s / 256 * 1e3,
                    "plain_per_set_ms": plain_ppr_s * 1e3,
                    "batched_vs_plain": plain_ppr_s * 256 / ppr_s,
                    "parity": ppr_parity}}


def leg_c4(W, O, torch, dev, stream, peak):
    """Lanczos: R-MAT 20 symmetrised, normalised Laplacian, 16 smallest;
    then the largest connected component (the full graph deflates)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    g = W.rmat(20, undirected=True)
    n, m = g.id_space, g.edges
    gv = g.upload()
    opts = W.EigenOptions(16, which="smallest", operator="normalized_laplacian", tol=1e-10,
                          max_iter=200, seed=7)
    W.eigen(gv, opts)
    t0 = time.perf_counter()
    e = W.eigen(gv, opts)
    full_s = time.perf_counter() - t0
    rows = np.repeat(np.arange(n), np.diff(g.offsets).astype(np.int64))
    a = csr_matrix((np.ones(m), (rows, g.targets)), shape=(n, n))
    _, labels = connected_components(a, directed=False)
    keep = np.where(labels == np.bincount(labels).argmax())[0]
    sub = a[keep][:, keep].tocsr()
    sub.sort_indices()
    gl = W.GraphVersion(sub.indptr.astype(np.uint64), sub.indices.astype(np.uint32))
    lopts = W.EigenOptions(16, which="smallest", operator="normalized_laplacian", tol=1e-10,
                           max_iter=4000, seed=7)
    W.eigen(gl, lopts)
    t0 = time.perf_counter()
    el = W.eigen(gl, lopts)
    lcc_s = time.perf_counter() - t0
    # An independent solver on the same component: ARPACK (scipy's eigsh)
    # on 2I - L, whose 16 largest eigenvalues are 2 minus the 16 smallest.
    from scipy.sparse import diags, identity
    from scipy.sparse.linalg import eigsh
    inv = diags(1.0 / np.sqrt(np.asarray(sub.sum(axis=1)).ravel()))
    t0 = time.perf_counter()
    ref = np.sort(2.0 - eigsh(identity(sub.shape[0]) + inv @ sub @ inv, k=16, which="LA",
                              ncv=96, tol=1e-14, maxiter=100000, return_eigenvectors=False))
    arpack_s = time.perf_counter() - t0
    return {"graph": {"scale": 20, "nodes": n, "stored_entries": m},
            "full": {"components": e.components, "exact_zeros": e.exact, "steps": e.iterations,
                     "seconds": full_s, "max_residual": float(e.residuals.max())},
            "largest_component": {"nodes": int(len(keep)), "stored_entries": int(sub.nnz),
                                  "steps": el.iterations, "converged": el.converged,
                                  "seconds": lcc_s,
                                  "ms_per_step": lcc_s / max(1, el.iterations) * 1e3,
                                  "max_residual": float(el.residuals.max()),
                                  "smallest": [float(v) for v in el.values[:4]],
                                  "vs_arpack_max_abs": float(np.abs(np.sort(el.values) - ref).max()),
                                  "arpack_seconds_cpu": arpack_s}}


def leg_c5(W, O, torch, dev, stream, peak):
    """PageRank adjoint: R-MAT 22, lognormal(0,1) row-normalised weights,
    64 losses of 1,000 random targets; central differences on a few edges."""
    g = W.rmat(22)
    n, m = g.id_space, g.edges
    w = W.edge_weights(g, "lognormal")
    gv = W.GraphVersion(g.offsets, g.targets, w)
    rng = np.random.default_rng(SEED)
    losses = [rng.choice(n, 1000, replace=False) for _ in range(64)]
    pr = W.PageRank(0.85, None, 100)
    grad = torch.empty((64, m), dtype=torch.float64, device=dev)
    W.pagerank_adjoint(gv, losses[:1], pr, adjoint_tol=1e-14, grad_out=grad[:1])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    _, ranks, its = W.pagerank_adjoint(gv, losses, pr, adjoint_tol=1e-14, grad_out=grad)
    torch.cuda.synchronize(dev)
    adj_s = time.perf_counter() - t0
    # Parity at this size: the oracle's FP64 CPU adjoint for the first loss.
    og = O.Graph.from_csr(n, g.offsets, g.targets, w)
    go, ro, ito = O.pagerank_adjoint(og, losses[:1], 0.85, None, 100, 1e-14)
    del og
    g0 = grad[0].cpu().numpy()
    adj_parity = {"checked_losses": 1,
                  "max_abs_diff_over_max_abs": float(np.abs(g0 - go[0]).max() / np.abs(go[0]).max()),
                  "ranks_rel_l1": float(np.abs(ranks - ro).sum() / ro.sum()),
                  "iterations_equal": bool(int(its[0]) == int(ito[0]) and int(its[1]) >= 1)}
    h = 1e-6
    checks = []
    for e in rng.choice(m, 3, replace=False):
        vals = []
        for sgn in (1, -1):
            wp = w.copy()
            wp[e] += sgn * h
            r = W.pagerank(W.GraphVersion(g.offsets, g.targets, wp), None, pr)
            vals.append(r.values[losses[0]].sum())
        fd = (vals[0] - vals[1]) / (2 * h)
        gd = float(grad[0, int(e)].item())
        floor = 1e-16 * vals[0] / h
        checks.append({"edge": int(e), "fd": fd, "adjoint": gd,
                       "within": bool(abs(fd - gd) <= 1e-6 * abs(gd) + 4 * floor),
                       "rel": abs(fd - gd) / max(abs(gd), 1e-300), "fd_floor": floor})
    return {"graph": {"scale": 22, "nodes": n, "edges": m}, "losses": 64,
            "targets_per_loss": 1000, "seconds": adj_s, "forward_iterations": int(its[0]),
            "adjoint_iterations": int(its[1]), "fd_checks": checks, "parity": adj_parity}


def leg_cent(W, O, torch, dev, stream, peak):
    """Closeness and harmonic centrality on the batched BFS (no reference
    configuration names them; R-MAT 22 and 16 as C1-C3): a seeded sample of
    1,024 sources on R-MAT 22, every node of R-MAT 16, and a 64-source
    sample checked bit for bit against the oracle, which also times it."""
    out = {}
    g = W.rmat(22)
    gv = g.upload()
    t0 = time.perf_counter()
    src = W.sample_sources(g.id_space, W.Sampling(k=1024, seed=7))
    sample_s = time.perf_counter() - t0
    W.closeness_centrality(gv, sources=src)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    c = W.closeness_centrality(gv, sources=src)
    t1 = time.perf_counter()
    W.harmonic_centrality(gv, sources=src)
    t2 = time.perf_counter()
    out["rmat22_sample1024"] = {"sources": c.sources, "sample_s": sample_s,
                                "closeness_s": t1 - t0, "harmonic_s": t2 - t1,
                                "source_edges_per_s": c.sources * g.edges / (t1 - t0)}
    del gv
    g16 = W.rmat(16)
    gv16 = g16.upload()
    every = W.sample_sources(g16.id_space)
    W.closeness_centrality(gv16, sources=every)
    t0 = time.perf_counter()
    c16 = W.closeness_centrality(gv16, sources=every)
    every_s = time.perf_counter() - t0
    og16 = O.Graph.from_csr(g16.id_space, g16.offsets, g16.targets)
    small = W.Sampling(k=64, seed=3)
    src = W.sample_sources(g16.id_space, small)
    t0 = time.perf_counter()
    want = O.centrality(og16, "harmonic", src)
    cpu_s = time.perf_counter() - t0
    got = W.harmonic_centrality(gv16, small).values
    out["rmat16_every_node"] = {"sources": c16.sources, "seconds": every_s,
                                "per_source_us": every_s / c16.sources * 1e6}
    # Betweenness (Brandes): 256 sampled sources on R-MAT 22, and a bit-for-bit
    # check with the oracle's per-source timing on 8 sources of R-MAT 16.
    gv = g.upload()
    bsrc = W.sample_sources(g.id_space, W.Sampling(k=256, seed=5))
    W.betweenness_centrality(gv, sources=bsrc[:64])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    W.betweenness_centrality(gv, sources=bsrc)
    bc_s = time.perf_counter() - t0
    del gv
    src8 = W.sample_sources(g16.id_space, W.Sampling(k=8, seed=2))
    t0 = time.perf_counter()
    bwant = O.betweenness(og16, src8)
    bc_cpu = time.perf_counter() - t0
    bgot = W.betweenness_centrality(gv16, sources=src8).values
    out["betweenness_rmat22_sample256"] = {"sources": 256, "seconds": bc_s,
                                           "per_source_ms": bc_s / 256 * 1e3}
    rel = np.abs(bgot - bwant) / np.maximum(np.abs(bwant), 1e-300)
    out["betweenness_rmat16_sample8"] = {"max_rel_diff_vs_oracle": float(rel[bwant != 0].max()),
                                         "rows_over_256_reassociated": True,
                                         "cpu_oracle_per_source_ms": bc_cpu / 8 * 1e3,
                                         "cpu_threads": 1}
    out["rmat16_sample64"] = {"bit_exact_vs_oracle": bool(got.tobytes() == want.tobytes()),
                              "cpu_oracle_s": cpu_s, "cpu_threads": 1,
                              "cpu_per_source_ms": cpu_s / 64 * 1e3}
    return out


def leg_load(W, O, torch, dev, stream, peak):
    """A version's device copy at R-MAT 22 (weighted, f64): from host arrays
    with the reverse CSR transposed on the device, with the reverse given
    (the host's counting transpose, timed apart), and from the stored CSR
    segments (dense and sparse offsets), checked on the device."""
    from pg_warren_b200 import api
    g = W.rmat(22)
    w = W.edge_weights(g, "uniform")
    out = {"nodes": g.id_space, "edges": g.edges}

    def timed(make):
        gv = make()
        del gv
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        gv = make()
        seconds = time.perf_counter() - t0
        del gv
        return seconds

    out["arrays_device_reverse_s"] = timed(lambda: W.GraphVersion(g.offsets, g.targets, w))
    t0 = time.perf_counter()
    rev = api.host_reverse(g.offsets, g.targets, w)
    out["host_transpose_s"] = time.perf_counter() - t0
    out["arrays_given_reverse_s"] = timed(lambda: W.GraphVersion(g.offsets, g.targets, w,
                                                                 reverse=rev))
    for sparse in (False, True):
        rows, off, tgt, ws = api.csr_segments(g.offsets, g.targets, w, sparse=sparse)
        key = "segments_sparse_s" if sparse else "segments_dense_s"
        out[key] = timed(lambda: W.GraphVersion.from_segments(g.id_space, off, tgt, ws, rows))
    return out


def suite(args):
    import torch
    import pg_warren_b200 as W
    import oracle as O
    O.build()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    peak, kind = measured_peaks()
    legs = {"c1": leg_c1, "c2": leg_c2, "c3": leg_c3, "c4": leg_c4, "c5": leg_c5,
            "cent": leg_cent, "load": leg_load}
    out = {"peak_gbs": peak, "peak_kind": kind}
    for name in args.suite.split(","):
        t0 = time.time()
        out[name] = legs[name](W, O, torch, dev, stream, peak)
        out[name]["wall_s"] = time.time() - t0
        torch.cuda.empty_cache()
    print(json.dumps(out))


# --------------------------------------------------------------- profiler cases
# `python bench.py --case batched|spmv|ppr|minplus|eigen|adjoint|bfspart|all --scale S`: one
# small workload per kernel family, for ncu captures (a few GB on the device
# at most).

def profile_case(args):
    import torch
    import pg_warren_b200 as W
    g = W.rmat(args.scale)
    gv = g.upload()
    n = g.id_space
    stream = torch.cuda.Stream()
    if args.case == "batched":
        # 1,024 sources, caps 16, one pass of 1,024 columns; two calls.
        rng = np.random.default_rng(SEED)
        src = torch.as_tensor(rng.integers(0, n, 1024).astype(np.int64), device="cuda")
        caps = torch.full((1024,), 16, dtype=torch.int32, device="cuda")
        W.set_schedule(gv, "bfs", 1024, columns_per_pass=1024, blocks_per_sm=8)
        d = torch.empty((1024, n), dtype=torch.uint8, device="cuda")
        e = torch.empty(1024, dtype=torch.int64, device="cuda")
        for _ in range(2):
            W.bfs_batched(gv, src, caps, depth_out=d, edges_out=e, stream=stream, timing=True)
            print(json.dumps({"level": gv.timing("level"), "depth": gv.timing("depth")}))
        torch.cuda.synchronize()
        print(json.dumps({"case": "batched", "nodes": n, "edges": g.edges,
                          "edges_traversed": int(e.sum())}))
    elif args.case == "ppr":
        # 32 personalised PageRank seed sets (sizes log-uniform 1..1000),
        # one pass of 32 columns, tol 1e-10; two calls.
        rng = np.random.default_rng(SEED)
        sizes = np.exp(rng.uniform(0, np.log(1000), 32)).astype(np.int64)
        sets = [rng.choice(n, int(s), replace=False) for s in sizes]
        W.set_schedule(gv, "ppr", 32, columns_per_pass=32, blocks_per_sm=5)
        r = torch.empty((32, n), dtype=torch.float64, device="cuda")
        it = torch.empty(32, dtype=torch.int32, device="cuda")
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            W.ppr_batched(gv, sets, W.PageRank(0.85, 1e-10, 100), ranks_out=r,
                          iterations_out=it)
            torch.cuda.synchronize()
            seconds = time.perf_counter() - t0
        print(json.dumps({"case": "ppr", "nodes": n, "edges": g.edges, "seconds": seconds,
                          "iterations_max": int(it.max()), "iterations_mean": float(it.float().mean())}))
    elif args.case == "minplus":
        # Batched min-plus: 1,024 sources, int32 weights 1..100, caps
        # U{1..16}, as the suite's C3 leg at a smaller scale; two calls.
        rng = np.random.default_rng(SEED)
        wi = rng.integers(1, 101, g.edges).astype(np.float64)
        gw = W.GraphVersion(g.offsets, g.targets, wi)
        src = rng.integers(0, n, 1024).astype(np.uint64)
        caps = rng.integers(1, 17, 1024).astype(np.uint32)
        d = torch.empty((1024, n), dtype=torch.int64, device="cuda")
        it = torch.empty(1024, dtype=torch.int32, device="cuda")
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            W.minplus_batched(gw, src, caps, dist_out=d, iterations_out=it)
            torch.cuda.synchronize()
            seconds = time.perf_counter() - t0
        print(json.dumps({"case": "minplus", "nodes": n, "edges": g.edges, "seconds": seconds,
                          "column_iterations": int(it.sum())}))
    elif args.case == "eigen":
        # Lanczos on the largest connected component of the symmetrised
        # R-MAT: normalised Laplacian, 16 smallest, as the suite's C4
        # variant at a smaller scale; two calls.
        from scipy.sparse import csr_matrix
        from scipy.sparse.csgraph import connected_components
        gs = W.rmat(args.scale, undirected=True)
        ns, ms = gs.id_space, gs.edges
        rows = np.repeat(np.arange(ns), np.diff(gs.offsets).astype(np.int64))
        a = csr_matrix((np.ones(ms), (rows, gs.targets)), shape=(ns, ns))
        _, labels = connected_components(a, directed=False)
        keep = np.where(labels == np.bincount(labels).argmax())[0]
        sub = a[keep][:, keep].tocsr()
        sub.sort_indices()
        gl = W.GraphVersion(sub.indptr.astype(np.uint64), sub.indices.astype(np.uint32))
        opts = W.EigenOptions(16, which="smallest", operator="normalized_laplacian", tol=1e-10,
                              max_iter=4000, seed=7)
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e = W.eigen(gl, opts)
            torch.cuda.synchronize()
            seconds = time.perf_counter() - t0
        print(json.dumps({"case": "eigen", "nodes": int(len(keep)), "entries": int(sub.nnz),
                          "seconds": seconds, "steps": int(e.iterations)}))
    elif args.case == "adjoint":
        # PageRank adjoint: lognormal(0,1) row-normalised weights, 64
        # losses of 1,000 random targets, as the suite's C5 leg at a smaller
        # scale; two calls.
        rng = np.random.default_rng(SEED)
        gw = W.GraphVersion(g.offsets, g.targets, W.edge_weights(g, "lognormal"))
        losses = [rng.choice(n, 1000, replace=False) for _ in range(64)]
        grad = torch.empty((64, g.edges), dtype=torch.float64, device="cuda")
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, _, its = W.pagerank_adjoint(gw, losses, W.PageRank(0.85, None, 100),
                                           adjoint_tol=1e-14, grad_out=grad)
            torch.cuda.synchronize()
            seconds = time.perf_counter() - t0
        print(json.dumps({"case": "adjoint", "nodes": n, "edges": g.edges, "seconds": seconds,
                          "iterations": [int(i) for i in its]}))
    elif args.case == "all":
        # Every kernel family once on the same graph, for a launch list with
        # each kernel's DRAM bytes: products in every element type, PageRank
        # (plain, seeded, no-allocation), the traversals (plain, visits,
        # reachable set, cursor, components), the batched searches, the
        # eigensolver, the adjoint, top-k, the vector map and reductions,
        # the centralities, the version load from segments and the
        # partitioned parts.
        from pg_warren_b200 import expr as X
        from pg_warren_b200.partition import bfs_partitioned, SpmvDeviceParts
        rng = np.random.default_rng(SEED)
        xf = torch.rand(n, dtype=torch.float64, device="cuda")
        for sr, dt in (("plus_times", torch.float64), ("plus_times", torch.float32),
                       ("min_plus", torch.int64), ("lor_land", torch.bool)):
            xx = (xf * 100).to(dt) if dt != torch.bool else xf < 0.1
            yy = torch.zeros(n, dtype=dt, device="cuda")
            W.spmv(gv, W.Product(sr, transpose=True), xx, yy)
        W.spmm(gv, W.Product("plus_times"), torch.rand((n, 8), dtype=torch.float64, device="cuda"),
               torch.zeros((n, 8), dtype=torch.float64, device="cuda"))
        W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100))
        seed = np.zeros(n)
        seed[rng.choice(n, 100, replace=False)] = 1.0
        W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100, seed=seed))
        W.pagerank_noalloc(gv, None, W.PageRank(0.85, 1e-10, 100))
        starts = [int(v) for v in rng.integers(0, n, 4)]
        W.bfs_depths(gv, starts)
        W.bfs(gv, starts[:1], limits=W.Limits(3, None))
        W.reachable_set(gv, starts, None, "both")
        cur = W.BfsCursor(gv, starts[:1])
        for _ in range(4):
            cur.next_level()
        cur.close()
        W.components(gv)
        src = torch.as_tensor(rng.integers(0, n, 256).astype(np.int64), device="cuda")
        caps = torch.full((256,), 16, dtype=torch.int32, device="cuda")
        W.bfs_batched(gv, src, caps)
        wi = rng.integers(1, 101, g.edges).astype(np.float64)
        gw = W.GraphVersion(g.offsets, g.targets, wi)
        W.minplus_batched(gw, rng.integers(0, n, 64).astype(np.uint64),
                          np.full(64, 8, np.uint32))
        sets = [rng.choice(n, int(k), replace=False) for k in rng.integers(1, 300, 32)]
        W.ppr_batched(gv, sets, W.PageRank(0.85, 1e-10, 100))
        gs = W.rmat(16, undirected=True).upload()
        W.eigen(gs, W.EigenOptions(4, which="smallest", operator="normalized_laplacian",
                                   tol=1e-8, max_iter=400, seed=7))
        gl = W.GraphVersion(g.offsets, g.targets, W.edge_weights(g, "lognormal"))
        W.pagerank_adjoint(gl, [rng.choice(n, 100, replace=False) for _ in range(4)],
                           W.PageRank(0.85, None, 20))
        W.top_k(gv, xf, 100)
        W.vector_map(gv, X.Arithmetic("+", X.Call("sqrt", X.Vector("f64", 0)),
                                      X.Literal("f64", 1.0)), [xf])
        W.vector_reduce(gv, xf, "sum")
        W.vector_norm_diff(gv, xf, xf * 0.5, "l1")
        W.closeness_centrality(gv, W.Sampling(k=64, seed=3))
        W.betweenness_centrality(gv, W.Sampling(k=16, seed=3))
        rows, offs, tgts, wts = W.api.csr_segments(g.offsets, g.targets)
        W.GraphVersion.from_segments(n, offs, tgts, wts, rows)
        bfs_partitioned(gv, starts[:1])
        SpmvDeviceParts(gv, W.Product("plus_times", transpose=True)).apply(
            2, 1, xf, torch.zeros_like(xf))
        torch.cuda.synchronize()
        print(json.dumps({"case": "all", "nodes": n, "edges": g.edges,
                          "launches": int(W.load().wc_kernel_launches())}))
    elif args.case == "bfspart":
        # The row-partitioned level search as one part (its pull, push and
        # settle kernels), from one seed, two calls; then one part of a
        # two-part product over the reverse CSR.
        from pg_warren_b200.partition import bfs_partitioned, SpmvDeviceParts
        seed = [int(np.random.default_rng(SEED).integers(0, n))]
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            depth, levels = bfs_partitioned(gv, seed)
            seconds = time.perf_counter() - t0
        x = torch.rand(n, dtype=torch.float64, device="cuda")
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        SpmvDeviceParts(gv, W.Product("plus_times", transpose=True)).apply(2, 0, x, y)
        torch.cuda.synchronize()
        print(json.dumps({"case": "bfspart", "nodes": n, "edges": g.edges, "levels": levels,
                          "reached": int((depth != 0xFFFFFFFF).sum()), "seconds": seconds}))
    else:
        # SpMV plus_times (f64, unweighted) over the forward CSR three
        # times, then a PageRank of three iterations.
        x = torch.rand(n, dtype=torch.float64, device="cuda")
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        for _ in range(3):
            W.spmv(gv, W.Product("plus_times"), x, y)
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        r = W.pagerank(gv, None, W.PageRank(0.85, None, 3), out=out)
        torch.cuda.synchronize()
        print(json.dumps({"case": "spmv", "nodes": n, "edges": g.edges,
                          "iterations": r.iterations}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="warren")
    ap.add_argument("--suite", default=None,
                    help="comma-separated configurations to measure instead: c1,c2,c3,c4,c5,cent,load")
    ap.add_argument("--case", default=None, choices=["batched", "spmv", "ppr", "minplus", "eigen", "adjoint",
                                                       "bfspart", "all"],
                    help="a small workload for profilers instead")
    ap.add_argument("--scale", type=int, default=20)
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.suite:
        return suite(args)
    if args.case:
        return profile_case(args)

    import torch
    import pg_warren_b200 as W

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    lib = W.load()
    peak, peak_kind = measured_peaks()

    g = make_graph()
    n, m = g.id_space, g.edges
    gv = g.upload()
    src, caps = sources_and_caps(n, rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()

    def reduce(x, op):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    # ---- batched: 1,024 searches, device-resident
    sched = W.autotune(gv, "bfs", WIDTH)
    columns = sched.columns_per_pass
    src_d = torch.as_tensor(src.view(np.int64), device=dev)
    caps_d = torch.as_tensor(caps.view(np.int32), device=dev)
    depth_d = torch.empty((WIDTH, n), dtype=torch.uint8, device=dev)
    edges_d = torch.empty(WIDTH, dtype=torch.int64, device=dev)

    def batched(timing=False):
        W.bfs_batched(gv, src_d, caps_d, depth_out=depth_d, edges_out=edges_d, stream=stream,
                      timing=timing)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            batched()
        torch.cuda.synchronize(dev)
        barrier()
        step_ms = []
        launches0 = lib.wc_kernel_launches()
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                flush.fill_(1)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                batched()
                b.record(stream)
                b.synchronize()
                step_ms.append(a.elapsed_time(b))
        launches = lib.wc_kernel_launches() - launches0
        barrier()
        # The kernel groups' times, from as many further steps made with the
        # library's events (kept out of the timed steps above).
        level_ms, level_launches, depth_ms, pull_ms, pulled = 0.0, 0, 0.0, 0.0, 0
        for _ in range(args.steps):
            flush.fill_(1)
            batched(timing=True)
            ms, nl = gv.timing("level")
            level_ms += ms
            level_launches += nl
            depth_ms += gv.timing("depth")[0]
            pull_ms += gv.timing("pull")[0]
            pulled += gv.timing("pulled")[1]
        torch.cuda.synchronize(dev)
    edges_step = int(edges_d.sum().item())
    total_ms = reduce(sum(step_ms), dist.ReduceOp.MAX if dist else None)
    edges_all = reduce(float(edges_step), dist.ReduceOp.SUM if dist else None)
    value = edges_all * args.steps / (total_ms * 1e-3) / 1e9
    batched_gteps_rank = edges_step * args.steps / (sum(step_ms) * 1e-3) / 1e9
    levels = executed_levels(depth_d, caps, columns)
    level_bytes = 4 * (n + 1) + 4 * m + n * columns // 4
    # The roofline of msbfs_level_kernel: its launches timed alone, over the
    # levels that pulled (the push levels' launches return at once).
    pulled_per_step = pulled / args.steps
    pull_avg_ms = pull_ms / pulled if pulled else None
    achieved = level_bytes / (pull_avg_ms * 1e-3) / 1e9 if pull_avg_ms else None

    # ---- plain per-source GPU path, a sample of the same sources
    dpl = torch.empty(n, dtype=torch.int32, device=dev)
    vpl = torch.empty(n, dtype=torch.int64, device=dev)
    for s, c in zip(src[:2], caps[:2]):
        W.bfs_depths(gv, [int(s)], max_depth=int(c), depth_out=dpl, via_out=vpl)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    plain_edges = 0
    for s, c in zip(src[:PLAIN_SAMPLE], caps[:PLAIN_SAMPLE]):
        _, _, st = W.bfs_depths(gv, [int(s)], max_depth=int(c), depth_out=dpl, via_out=vpl)
        plain_edges += st.edges_traversed
    torch.cuda.synchronize(dev)
    plain_gteps = plain_edges / (time.perf_counter() - t0) / 1e9

    # ---- PageRank (FP64, uniform), iterations/s
    ranks_d = torch.empty(n, dtype=torch.float64, device=dev)
    opts = W.PageRank(0.85, 1e-10, 100)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            W.pagerank(gv, None, opts, out=ranks_d, stream=stream)
        torch.cuda.synchronize(dev)
        pr_ms, pr_it, pr_iter_ms = [], 0, 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r = W.pagerank(gv, None, opts, out=ranks_d, stream=stream, timing=True)
            b.record(stream)
            b.synchronize()
            pr_ms.append(a.elapsed_time(b))
            pr_it = r.iterations
            pr_iter_ms += gv.timing("iteration")[0]
    pr_bytes = 4 * (n + 1) + 4 * m + 24 * n
    pr_kernel_gbs = pr_bytes * pr_it * args.steps / (pr_iter_ms * 1e-3) / 1e9 if pr_iter_ms else 0.0
    pagerank = {"iterations": pr_it, "ms": statistics.median(pr_ms),
                "iters_per_s": pr_it / (statistics.median(pr_ms) * 1e-3),
                "roofline": {"bound": "hbm", "kernel": "pr_iter_kernel",
                             "achieved": pr_kernel_gbs, "peak": peak, "unit": "GB/s",
                             "frac": pr_kernel_gbs / peak,
                             "bytes_per_iteration": pr_bytes}}

    # ---- beside the headline: the SpMV's fraction, the batched min-plus
    # and personalised PageRank against their plain per-source paths (the
    # batched-traversal configuration's other two workloads)
    spmv = spmv_point(W, torch, dev, stream, peak, g)
    # The oracle checks the batched min-plus (8 sources) and personalised
    # PageRank (3 sets) outputs at this size, outside their timed calls, on
    # rank 0 of a one-GPU run (as the CPU baseline below checks the depths).
    checker = None
    if rank == 0 and world == 1:
        import oracle as checker
        checker.build()
    c3 = leg_c3(W, checker, torch, dev, stream, peak, g=g)
    torch.cuda.empty_cache()

    # ---- end to end through the public call, host buffers
    src_h = torch.from_numpy(src.view(np.int64)).pin_memory()
    caps_h = torch.from_numpy(caps.view(np.int32)).pin_memory()
    depth_h = torch.empty((WIDTH, n), dtype=torch.uint8, pin_memory=True)
    edges_h = torch.empty(WIDTH, dtype=torch.int64, pin_memory=True)
    W.bfs_batched(gv, src_h, caps_h, depth_out=depth_h, edges_out=edges_h, stream=stream)
    barrier()
    e2e_s = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        W.bfs_batched(gv, src_h, caps_h, depth_out=depth_h, edges_out=edges_h, stream=stream)
        e2e_s.append(time.perf_counter() - t0)
    e2e_total = reduce(sum(e2e_s), dist.ReduceOp.MAX if dist else None)
    e2e_value = edges_all * args.steps / e2e_total / 1e9
    assert int(edges_h.sum()) == edges_step, "host and device runs disagree"

    # ---- CPU baseline (rank 0, one GPU only), which also checks parity:
    # each sampled search's depths and edge count from the oracle against
    # the same source's row of the device-resident run and of the run with
    # host buffers, byte for byte.
    cpu, parity = None, None
    if rank == 0 and world == 1:
        mismatches = []

        def check(sl, d, e):
            dev_rows = depth_d[sl].cpu().numpy()
            if not (np.array_equal(d, dev_rows) and np.array_equal(d, depth_h[sl].numpy())
                    and np.array_equal(e.astype(np.int64), edges_d[sl].cpu().numpy())
                    and np.array_equal(e.astype(np.int64), edges_h[sl].numpy())):
                mismatches.append(sl.start)

        gt, done, threads, secs = cpu_bfs(g.offsets, g.targets, src, caps, CPU_BUDGET_S, check)
        cpu = {"value": gt, "unit": "GTEPS", "cores": threads, "kind": "port",
               "sample": f"{done} of the {WIDTH} searches, 64 a word (the reference's batched "
                         f"multi_source shape, {threads} threads, {secs:.1f} s)"}
        pgt, pdone, _, psecs = cpu_bfs(g.offsets, g.targets, src, caps, CPU_BUDGET_S / 2, None,
                                       batched=False)
        cpu["per_source"] = {"value": pgt, "unit": "GTEPS", "cores": threads,
                             "sample": f"{pdone} of the searches, one LevelSearch each, "
                                       f"{threads} at a time ({psecs:.1f} s)"}
        parity = {"checked_sources": done, "of": WIDTH, "bit_exact": not mismatches,
                  "compared": "depth bytes and edges_traversed of each sampled source, "
                              "device-resident and host-buffer runs, against the oracle"}

    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": config(n, m),
        "schedule": {"columns_per_pass": columns, "blocks_per_sm": sched.blocks_per_sm},
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": WIDTH * 12,
                "d2h_bytes_per_step": WIDTH * n + WIDTH * 8},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None,
                     "traffic": level_bytes * LEVEL_TRAFFIC_RATIO,
                     "traffic_source": LEVEL_TRAFFIC_SOURCE,
                     "kernel": "msbfs_level_kernel",
                     "bytes_per_level": level_bytes, "pulled_levels_per_step": pulled_per_step,
                     "levels_per_step": levels, "pull_ms_avg": pull_avg_ms,
                     "peak_kind": peak_kind,
                     "pull_ms_per_step": pull_ms / args.steps,
                     "level_ms_per_step": level_ms / args.steps,
                     "depth_ms_per_step": depth_ms / args.steps},
        "cpu_baseline": cpu,
        "parity": parity,
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "edges_traversed_per_step": edges_step,
        "batched_gteps_rank0": batched_gteps_rank,
        "plain_bfs_gteps": plain_gteps,
        "batched_vs_plain": batched_gteps_rank / plain_gteps,
        "pagerank_iters_per_s": pagerank["iters_per_s"],
        "pagerank": pagerank,
        "spmv": spmv,
        "minplus_batched": c3["minplus"],
        "ppr_batched": c3["ppr"],
    }
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
