#!/usr/bin/env python
"""Benchmark of the in-HBM hot path: PageRank + SSSP on a seeded R-MAT graph.

Workload (default): R-MAT scale 24, edge factor 16 (a,b,c = .57,.19,.19,
uint32 weights uniform [1,63], self-loops/duplicates removed), graph
resident in HBM, stored in the reference's hub order (HubSorter ranking,
built at graph creation; sources and results in the generator's ids;
--vertex-order input keeps the generator's order).  One step = PageRank (damping 0.85) to L1 change <= 1e-6
(max 100 iterations) + SSSP from 8 seeded sources, one at a time.

Metric: GTEPS = traversed edges / s, with E per PageRank iteration and E per
SSSP source (Graph500 convention), summed over all ranks (weak scaling:
every rank solves its own replica; the path has no cross-rank exchange).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PR/SSSP GTEPS (in/out-of-HBM) + served queries/s & p99 vs one-at-a-time"
UNIT = "GTEPS"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--sources", type=int, default=8)
    ap.add_argument("--seed", type=int, default=20241203)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the timed run's results")
    ap.add_argument("--workload", choices=["inhbm", "hybrid", "batch", "serve", "hubsort", "load", "contrib",
                                           "ppr8", "shard"],
                    default="inhbm",
                    help="inhbm: graph resident in HBM (default); hybrid: edges in pinned host memory under a "
                         "device budget (defaults to R-MAT scale 27, edge factor 32, 8 GiB); batch: 64 graphs of "
                         "scales 12-20, 512 SSSP/PPR queries in one CUDA-graph launch; serve: continuous "
                         "batching of a Poisson stream; hubsort: hub sorting + vertex reordering of the graph; load: "
                         "text edge list -> CSR in HBM (GraphLoader) and the binary CSR file; contrib: PageRank "
                         "contributions + contribution schedule of every vertex + partition priorities; ppr8: 8 personalized "
                         "PageRank queries packed into one solve vs one at a time; shard: the inhbm step on ONE graph "
                         "split by vertex range over all ranks (strong scaling, vectors exchanged over NCCL)")
    ap.add_argument("--hub-fraction", type=float, default=0.08)
    ap.add_argument("--vertex-order", choices=["input", "hub"], default="hub",
                    help="inhbm: store the graph in hub order (HYT_GRAPH_HUB_ORDER); results stay in input ids")
    ap.add_argument("--text-scale", type=int, default=22, help="load: R-MAT scale of the text edge list")
    ap.add_argument("--no-effect", action="store_true", help="hubsort: skip the solver comparison")
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--rates", type=str, default="200,500,1000,2000,5000")
    ap.add_argument("--rate-seconds", type=float, default=8.0, help="serve: cap on each rate point's duration")
    ap.add_argument("--graphs", type=int, default=64)
    ap.add_argument("--queries", type=int, default=512)
    ap.add_argument("--budget-gib", type=float, default=8.0)
    ap.add_argument("--partition-vertices", type=int, default=1 << 20)
    a = ap.parse_args()
    if a.workload == "hybrid":
        if "--scale" not in sys.argv:
            a.scale = 27
        if "--edge-factor" not in sys.argv:
            a.edge_factor = 32
    return a


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.out = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas, no data-path exchange)
# --------------------------------------------------------------------------
def dist_setup(gpus: int):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if gpus > 1 and world == 1:
        raise SystemExit("--gpus > 1 needs torchrun (one process per GPU)")
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local, pg


def barrier(pg):
    import torch

    if pg is not None:
        pg.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(pg, x: float) -> float:
    """Max of a per-rank timing over all ranks (NCCL on GPUs; any backend)."""
    import torch

    if pg is None:
        return x
    on_gpu = pg.get_backend() == "nccl"
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if on_gpu else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, world: int, ms_max: float) -> float:
    """Whole-job throughput of weak-scaled replicas: every rank processes
    units_per_rank, the job takes the slowest rank's time."""
    return units_per_rank * world / (ms_max / 1e3)


# --------------------------------------------------------------------------
# CPU side: the reference's own CPU solvers (oracle/_ref) timed with the GPU
# arm's counting convention, and the parity checks against the oracle.
# --------------------------------------------------------------------------
class CpuSolvers:
    """pagerank_cpu / sssp_cpu of the reference compiled from its sources
    (oracle/_ref, single-threaded as in the reference), or the oracle's
    restatements when _ref is absent."""

    def __init__(self):
        from oracle.bindings import Oracle, Reference

        if Reference.available():
            r = Reference()
            self.kind, self.cores = "reference", 1
            self.pagerank = lambda off, cols, it: r.pagerank_cpu(off, cols, 0.85, 1e-6, it)
            self.sssp = lambda off, cols, w, s, it: r.sssp_cpu(off, cols, w, int(s), it)
        else:
            o = Oracle()
            self.kind, self.cores = "port", int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))
            self.pagerank = lambda off, cols, it: o.pagerank_f32(off, cols, 0.85, 1e-6, it)
            self.sssp = lambda off, cols, w, s, it: o.sssp(off, cols, w, int(s), it)


def time_call(f, *a):
    t0 = time.perf_counter()
    r = f(*a)
    return time.perf_counter() - t0, r


def host_rmat(args):
    """The bench graph and its sources built on the host by the oracle's
    restatement of the generator (byte-identical to the product's; the
    reference arm loads no product library)."""
    from oracle.bindings import Oracle

    o = Oracle()
    off, cols, w = o.rmat(args.scale, args.edge_factor, args.seed)
    return off, cols, w, [int(x) for x in o.pick_sources(off, args.seed, args.sources)]


def project_step(parts, n_sources):
    """Full-solve step time (PageRank to convergence + n_sources SSSP solves)
    projected from one sampled first iteration / first round (each with its
    incoming-CSR build) plus the per-iteration and per-round costs."""
    pr = parts["pr_first_s"] + (parts["pr_iterations"] - 1) * parts["pr_per_iteration_s"]
    ss = parts["sssp_first_s"] + (parts["sssp_rounds"] - 1) * parts["sssp_per_round_s"]
    return pr + n_sources * ss


def cpu_baseline_sample(cpu, off, cols, w_f32, source, pr_iterations, sssp_rounds, n_sources):
    """Bounded CPU baseline on the full graph: pagerank_cpu for 1 and 3
    iterations and sssp_cpu for 1 and 3 rounds give the first-iteration and
    per-iteration costs; the iteration / round counts of the full solves come
    from the oracle's restatements, which reproduce the reference's counts
    bit for bit.  Returns (projected full-step seconds, parts, sample seconds)."""
    t_p1, _ = time_call(cpu.pagerank, off, cols, 1)
    t_p3, _ = time_call(cpu.pagerank, off, cols, 3)
    t_s1, _ = time_call(cpu.sssp, off, cols, w_f32, source, 1)
    t_s3, _ = time_call(cpu.sssp, off, cols, w_f32, source, 3)
    parts = {"pr_first_s": t_p1, "pr_per_iteration_s": max(t_p3 - t_p1, 0.0) / 2, "pr_iterations": pr_iterations,
             "sssp_first_s": t_s1, "sssp_per_round_s": max(t_s3 - t_s1, 0.0) / 2, "sssp_rounds": sssp_rounds}
    return project_step(parts, n_sources), parts, t_p1 + t_p3 + t_s1 + t_s3


def parity_inhbm(off, cols, w, sources, ranks, dists, threads=None):
    """The GPU results of the timed run against the oracle on the same graph:
    PageRank L1 against the FP64 restatement (and the reference's FP32
    solver's own L1, for context), SSSP labels of every source against
    Dijkstra (exact 64-bit integers), cross-checked on the first source with
    the restatement of the reference's synchronous Bellman-Ford."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.bindings import Oracle

    o = Oracle()
    w_f32 = w.astype(np.float32)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads or (len(sources) + 3)) as ex:
        f64 = ex.submit(o.pagerank_f64, off, cols, 0.85, 1e-6, 100)
        f32 = ex.submit(o.pagerank_f32, off, cols, 0.85, 1e-6, 100)
        bf = ex.submit(o.sssp, off, cols, w_f32, sources[0], 0)
        dj = [ex.submit(o.dijkstra, off, cols, w, s) for s in sources]
        r64, it64, _, _ = f64.result()
        r32, it32, _, _ = f32.result()
        want = []
        for d in dj:
            x = d.result()
            want.append(np.where(x == np.iinfo(np.uint64).max, 0xFFFFFFFF, x).astype(np.uint32))
        dbf, rounds_bf, _ = bf.result()
    mism = [int(np.count_nonzero(np.asarray(g).view(np.uint32) != x)) for g, x in zip(dists, want)]
    bf_u32 = np.where(np.isfinite(dbf), np.nan_to_num(dbf, posinf=0), 0).astype(np.uint32)
    bf_u32[~np.isfinite(dbf)] = 0xFFFFFFFF
    l1 = float(np.abs(np.asarray(ranks, np.float64) - r64).sum())
    return {"pr_l1_vs_fp64": l1, "pr_l1_ref_fp32_vs_fp64": float(np.abs(r32.astype(np.float64) - r64).sum()),
            "pr_l1_tolerance": 1e-5, "fp64_iterations": int(it64), "ref_fp32_iterations": int(it32),
            "sssp_mismatches": int(sum(mism)), "sources_checked": len(sources),
            "sssp_oracle": "Dijkstra, exact u64 labels, every source",
            "sssp_bellman_ford_vs_dijkstra_mismatches": int(np.count_nonzero(bf_u32 != want[0])),
            "ok": bool(l1 <= 1e-5 and sum(mism) == 0), "check_s": time.perf_counter() - t0,
            "_ref_rounds_source0": int(rounds_bf), "_ref_iterations": int(it32)}


def host_graph_from_device(dcsr):
    """Pinned host copy of a device-generated CSR (setup, not timed)."""
    import torch

    V, E = dcsr.num_vertices, dcsr.num_edges
    off = torch.empty(V + 1, dtype=torch.int64, pin_memory=True)
    cols = torch.empty(E, dtype=torch.int32, pin_memory=True)
    w = torch.empty(E, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    dcsr.download(off.numpy().view(np.uint64), cols.numpy().view(np.uint32), w.numpy().view(np.uint32))
    return off, cols, w


# --------------------------------------------------------------------------
def run_reference_arm(args, rank, pg):
    """--impl reference: the reference's CPU implementation of the path on
    this host's cores, same workload, metric, unit and counting convention
    (rank 0 only).  Only oracle/ libraries are loaded: the graph comes from
    the oracle's restatement of the generator."""
    if rank != 0:
        return
    if args.workload == "hubsort":
        off, cols, w, _ = host_rmat(args)
        V, E = int(off.shape[0] - 1), int(cols.shape[0])
        times, kind = [], "port"
        for i in range(args.warmup + args.steps):
            t, kind = reference_hubsort(off, cols, w, args.hub_fraction)
            if i >= args.warmup:
                times.append(t)
        total = sum(times)
        value = E * args.steps / total / 1e9
        sample = "per step: one HubSorter::sort + CSRGraph::reorder_vertices of the full graph"
        line = {"impl": "reference", "metric": "hub sort + reorder throughput", "value": value, "unit": "Gedges/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u32/u64 (f64 scores)", "data": "synthetic",
                "config": hubsort_config(args, V, E),
                "cpu_baseline": {"value": value, "unit": "Gedges/s", "cores": 1, "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": "Gedges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    t_gen = time.perf_counter()
    off, cols, w, sources = host_rmat(args)
    t_gen = time.perf_counter() - t_gen
    w_f32 = w.astype(np.float32)
    V, E = int(off.shape[0] - 1), int(cols.shape[0])
    cpu = CpuSolvers()
    n_src = len(sources)
    # Once, before the warm-up: the full solves give the iteration and round
    # counts and, with the per-step samples, the per-iteration costs.
    t_pr_full, (_, n_pr, _, _) = time_call(cpu.pagerank, off, cols, 100)
    t_ss_full, (_, n_ss, _) = time_call(cpu.sssp, off, cols, w_f32, sources[0], 0)
    samples = []
    for i in range(args.warmup + args.steps):
        t_p1, _ = time_call(cpu.pagerank, off, cols, 1)
        t_s1, _ = time_call(cpu.sssp, off, cols, w_f32, sources[0], 1)
        samples.append((t_p1, t_s1))
    med_p1 = statistics.median(x[0] for x in samples)
    med_s1 = statistics.median(x[1] for x in samples)
    per_it = max(t_pr_full - med_p1, 0.0) / max(n_pr - 1, 1)
    per_rd = max(t_ss_full - med_s1, 0.0) / max(n_ss - 1, 1)
    steps = []
    for t_p1, t_s1 in samples[args.warmup:]:
        steps.append(project_step({"pr_first_s": t_p1, "pr_per_iteration_s": per_it, "pr_iterations": n_pr,
                                   "sssp_first_s": t_s1, "sssp_per_round_s": per_rd, "sssp_rounds": n_ss}, n_src))
    total = sum(steps)
    traversed = args.steps * (E * n_pr + E * n_src)  # E per PageRank iteration + E per SSSP source
    value = traversed / total / 1e9
    parts = {"pr_full_s": t_pr_full, "pr_iterations": n_pr, "pr_first_iteration_s_median": med_p1,
             "pr_per_iteration_s": per_it, "sssp_full_s": t_ss_full, "sssp_rounds": n_ss,
             "sssp_first_round_s_median": med_s1, "sssp_per_round_s": per_rd, "graph_generation_s": t_gen}
    sample = (f"once: a full pagerank_cpu ({n_pr} iterations, {t_pr_full:.1f} s) and a full sssp_cpu from the "
              f"first source ({n_ss} rounds, {t_ss_full:.1f} s); per step: pagerank_cpu for 1 iteration and "
              f"sssp_cpu for 1 round (each with its incoming-CSR build) on the full R-MAT s{args.scale} "
              f"ef{args.edge_factor} graph; step time projected to PageRank to convergence + {n_src} full SSSP "
              f"solves (the first source's round count for each), E counted per PageRank iteration and per SSSP "
              f"source as in the GPU arm; single-threaded (the reference has no threads)")
    shard = args.workload == "shard"  # the same CPU work; the shard arm's metric and config
    line = {"impl": "reference", "metric": SHARD_METRIC if shard else METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "strong" if shard else "weak", "vs_baseline": None,
            "dtype": "f32/u32", "data": "synthetic",
            "config": shard_config(args, V, E, args.gpus) if shard else workload_config(args, V, E),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu.cores, "kind": cpu.kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "projection": {"parts": parts, "step_s": steps}}
    print(json.dumps(line), flush=True)


def run_hybrid(args, rank, world, pg):
    """Out-of-HBM workload: edges in pinned host memory, a device budget for
    edge data, partitions of --partition-vertices.  The graph is generated on
    the GPU, solved once in HBM (the parity reference at full size), copied
    to pinned host memory, and then solved by the hybrid engine: PageRank to
    L1 <= 1e-6 on a pull handle and SSSP from one seeded source on a push
    handle, each under the full budget."""
    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    peak_gbs, peak_kind = load_peaks()
    dcsr = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = dcsr.num_vertices, dcsr.num_edges
    b = dcsr.buffers
    off = hyt.PinnedBuffer(V + 1, np.uint64)
    cols = hyt.PinnedBuffer(E, np.uint32)
    w = hyt.PinnedBuffer(E, np.uint32)
    capi.copy(off.data_ptr(), C.cast(b.row_offsets, C.c_void_p).value, (V + 1) * 8)
    capi.copy(cols.data_ptr(), C.cast(b.column_indices, C.c_void_p).value, E * 4)
    capi.copy(w.data_ptr(), C.cast(b.weights, C.c_void_p).value, E * 4)
    src = int(hyt.pick_sources(off.array, args.seed, 1)[0])
    in_off = hyt.PinnedBuffer(V + 1, np.uint64)
    in_src = hyt.PinnedBuffer(E, np.uint32)

    # in-HBM solves of the same graph: full-size parity reference + context
    with hyt.Graph(dcsr, flags=capi.HYT_GRAPH_PULL) as g:
        g.copy_csc(in_off, in_src)
        ranks_hbm, pr_hbm = g.pagerank()
    with hyt.Graph(dcsr, flags=capi.HYT_GRAPH_PUSH) as g:
        dist_hbm, ss_hbm = g.sssp(src)
    dcsr.free()

    budget = int(args.budget_gib * (1 << 30))
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    with hyt.HybridGraph(off, cols, w, in_off, in_src, flags=capi.HYT_GRAPH_PULL, budget_bytes=budget,
                         partition_vertices=args.partition_vertices) as hp:
        pinfo = hp.info()
        clocks.start()
        t0 = time.perf_counter()
        ranks, pr, prt = hp.pagerank()
        pr_wall = time.perf_counter() - t0
    with hyt.HybridGraph(off, cols, w, flags=capi.HYT_GRAPH_PUSH, budget_bytes=budget,
                         partition_vertices=args.partition_vertices) as hs:
        sinfo = hs.info()
        t0 = time.perf_counter()
        dist, ss, sst = hs.sssp(src)
        ss_wall = time.perf_counter() - t0
    clk = clocks.stop()

    pr_l1 = float(np.abs(ranks.astype(np.float64) - ranks_hbm.astype(np.float64)).sum())
    sssp_equal = bool(np.array_equal(dist, dist_hbm))
    # parity against the oracle on the same host arrays: PageRank against
    # the FP64 restatement (on the CSC already in host memory), SSSP against
    # Dijkstra for the source
    parity = None
    if rank == 0 and not args.no_parity:
        from concurrent.futures import ThreadPoolExecutor

        from oracle.bindings import Oracle

        o = Oracle()
        t0 = time.perf_counter()
        with ThreadPoolExecutor(2) as ex:
            f64 = ex.submit(o.pagerank_f64_csc, off.array, in_off.array, in_src.array, 0.85, 1e-6, 100)
            dj = ex.submit(o.dijkstra, off.array, cols.array, w.array, src)
            r64, it64, _, _ = f64.result()
            d = dj.result()
        want = np.where(d == np.iinfo(np.uint64).max, 0xFFFFFFFF, d).astype(np.uint32)
        l1 = float(np.abs(ranks.astype(np.float64) - r64).sum())
        mism = int(np.count_nonzero(np.asarray(dist).view(np.uint32) != want))
        parity = {"pr_l1_vs_fp64": l1, "pr_l1_tolerance": 1e-5, "fp64_iterations": int(it64),
                  "sssp_mismatches": mism, "sources_checked": 1,
                  "sssp_oracle": "Dijkstra, exact u64 labels", "ok": bool(l1 <= 1e-5 and mism == 0),
                  "check_s": time.perf_counter() - t0}
    ms = pr["device_ms"] + ss["device_ms"]
    traversed = E * pr["iterations"] + E
    value = traversed / (ms / 1e3) / 1e9

    def link(st, t, info):
        bound_ms = t["necessary_bytes"] / (t["h2d_peak_gbs"] * 1e9) * 1e3
        return {"link_bytes": t["link_bytes"], "link_gbs": t["link_gbs"], "h2d_peak_gbs": t["h2d_peak_gbs"],
                "link_frac_of_peak": t["link_gbs"] / t["h2d_peak_gbs"],
                "necessary_bytes": t["necessary_bytes"], "host_link_bound_ms": bound_ms,
                "frac_of_host_link_bound": bound_ms / st["device_ms"],
                "filter_bytes": t["filter_bytes"], "compaction_bytes": t["compaction_bytes"],
                "zero_copy_bytes": t["zero_copy_bytes"], "copies": t["copies"],
                "decisions": {k: t[k + "_decisions"] for k in ("resident", "filter", "compaction", "zero_copy")},
                "compaction_host_ms": t["compaction_host_ms"],
                "resident_bytes": info["resident_bytes"], "staging_bytes": info["staging_bytes"],
                "device_bytes": info["device_bytes"], "zero_copy_gbs": info["zero_copy_gbs"],
                "gather_gbs": info["gather_gbs"]}

    pr_link, ss_link = link(pr, prt, pinfo), link(ss, sst, sinfo)
    frac = (pr_link["host_link_bound_ms"] + ss_link["host_link_bound_ms"]) / ms
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 0,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (PageRank) / u32 (SSSP)", "data": "synthetic",
                "config": {"workload": f"out-of-HBM hybrid transfer, R-MAT scale {args.scale} edge factor "
                                       f"{args.edge_factor}, edges in pinned host memory, device budget "
                                       f"{args.budget_gib:g} GiB, partitions of {args.partition_vertices} vertices: "
                                       f"PageRank to L1<=1e-6 + SSSP from 1 seeded source",
                           "scale": args.scale, "edge_factor": args.edge_factor, "vertices": V, "edges": E,
                           "budget_bytes": budget, "partitions": pinfo["partitions"], "seed": args.seed,
                           "host_bytes": (V + 1) * 16 + E * 12},
                "roofline": {"bound": "host-link", "achieved": (prt["link_bytes"] + sst["link_bytes"]) / (ms / 1e3) / 1e9,
                             "peak": prt["h2d_peak_gbs"], "unit": "GB/s",
                             "frac": frac, "frac_definition": "(necessary non-resident edge bytes / measured pinned "
                                                              "H2D peak) / measured solve time",
                             "hbm_peak_gbs": peak_gbs, "hbm_peak_kind": peak_kind},
                "pagerank": {"iterations": pr["iterations"], "ms": pr["device_ms"], "wall_s": pr_wall,
                             "gteps": E * pr["iterations"] / (pr["device_ms"] / 1e3) / 1e9,
                             "l1_vs_in_hbm": pr_l1, "in_hbm_ms": pr_hbm["device_ms"], **pr_link},
                "sssp": {"source": src, "rounds": ss["iterations"], "ms": ss["device_ms"], "wall_s": ss_wall,
                         "gteps": E / (ss["device_ms"] / 1e3) / 1e9, "identical_to_in_hbm": sssp_equal,
                         "in_hbm_ms": ss_hbm["device_ms"], **ss_link},
                "parity": parity, "clocks": clk, "gpu_launches": pr["total_launches"] + ss["total_launches"]}
        print(json.dumps(line), flush=True)
    for x in (off, cols, w, in_off, in_src):
        x.free()
    if not sssp_equal or pr_l1 > 1e-5:
        raise SystemExit(f"hybrid results differ from the in-HBM solve: sssp_equal={sssp_equal} pr_l1={pr_l1}")


def batch_workload(hyt, num_graphs, num_queries, seed, smin=12, smax=20, efmin=8, efmax=32):
    """Seeded uneven batch: graph scales U{smin..smax}, edge factors
    U{efmin..efmax}; 1-16 sources per graph adjusted to num_queries in
    total; each query SSSP with probability 0.6, else PPR (restart 0.15,
    tol 1e-6).  Returns (graph specs, queries)."""
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(smin, smax + 1)), int(rng.integers(efmin, efmax + 1)), int(seed + 1000 + i))
             for i in range(num_graphs)]
    counts = rng.integers(1, 17, num_graphs)
    while counts.sum() != num_queries:
        i = int(rng.integers(0, num_graphs))
        if counts.sum() > num_queries and counts[i] > 1:
            counts[i] -= 1
        elif counts.sum() < num_queries and counts[i] < 16:
            counts[i] += 1
    return specs, counts, rng


def run_batch_workload(args, rank, world, pg):
    """Batched uneven queries: every query of the batch in one
    hyt_batch_run (one CUDA-graph launch), against the same queries solved
    one at a time with hyt_sssp / hyt_ppr on the same graphs."""
    import torch
    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    specs, counts, rng = batch_workload(hyt, args.graphs, args.queries, args.seed)
    graphs, queries = [], []
    gflags = capi.HYT_GRAPH_ALL | (capi.HYT_GRAPH_HUB_ORDER if args.vertex_order == "hub" else 0)
    for gi, (sc, ef, gseed) in enumerate(specs):
        d = hyt.rmat(sc, ef, gseed, device=True)
        off = np.empty(d.num_vertices + 1, np.uint64)
        capi.copy(off.ctypes.data, C.cast(d.buffers.row_offsets, C.c_void_p).value, off.nbytes)
        graphs.append(hyt.Graph(d, flags=gflags))
        d.free()
        for s in hyt.pick_sources(off, gseed, int(counts[gi])):
            kind = "sssp" if rng.random() < 0.6 else "ppr"
            queries.append({"graph": gi, "kind": kind, "source": int(s), "restart": 0.15, "tolerance": 1e-6})
    E_of = [g.num_edges for g in graphs]
    V_of = [g.num_vertices for g in graphs]
    # device outputs (the bench line); pinned host outputs (e2e)
    dev_out = [torch.empty(V_of[q["graph"]], dtype=torch.int32 if q["kind"] == "sssp" else torch.float32,
                           device="cuda") for q in queries]
    host_out = [torch.empty(V_of[q["graph"]], dtype=torch.int32 if q["kind"] == "sssp" else torch.float32,
                            pin_memory=True) for q in queries]
    qd = [dict(q, out=o) for q, o in zip(queries, dev_out)]
    qh = [dict(q, out=o) for q, o in zip(queries, host_out)]
    torch.cuda.synchronize()
    with hyt.Batch(graphs) as b:
        t0 = time.perf_counter()
        tuning = b.autotune(queries)
        tune_s = time.perf_counter() - t0
        for _ in range(args.warmup):
            b.run(qd)
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        barrier(pg)
        ms_list, res, st = [], None, None
        for _ in range(args.steps):
            _, res, st = b.run(qd)
            ms_list.append(st["device_ms"])
        clk = clocks.stop()
        ms = max_over_ranks(pg, sum(ms_list) / len(ms_list))
        # e2e: results land in pinned host memory inside the timed call
        b.run(qh)
        t0 = time.perf_counter()
        _, _, st_h = b.run(qh)
        e2e_wall = time.perf_counter() - t0
    traversed = sum(E_of[q["graph"]] * (r["iterations"] if q["kind"] == "ppr" else 1) for q, r in zip(queries, res))
    n_q = len(queries)
    # a sample of the timed batch's results, checked against the oracle below
    torch.cuda.synchronize()
    sample_idx = list(range(0, n_q, max(1, n_q // 16)))[:16]
    sample_out = {i: dev_out[i].cpu().numpy().copy() for i in sample_idx}
    # one at a time: the same queries through hyt_sssp / hyt_ppr, outputs on
    # the device; every graph's solver state is allocated before timing
    for gi, g in enumerate(graphs):
        src = next(q["source"] for q in queries if q["graph"] == gi)
        o = torch.empty(V_of[gi], dtype=torch.float32, device="cuda")
        g.sssp(src, out=o.view(torch.int32))
        g.ppr(src, out=o)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for q, o in zip(queries, dev_out):
        g = graphs[q["graph"]]
        (g.sssp(q["source"], out=o) if q["kind"] == "sssp" else g.ppr(q["source"], out=o))
    e1.record()
    e1.synchronize()
    single_ms = e0.elapsed_time(e1)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = batch_cpu_sample(hyt, specs, queries)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = query_parity(specs, queries, sample_out)
    if rank == 0:
        gteps = traversed * world / (ms / 1e3) / 1e9
        line = {"metric": METRIC, "value": gteps, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (PPR) / u32 (SSSP)", "data": "synthetic",
                "config": {"workload": f"batched uneven queries: {len(graphs)} R-MAT graphs, scales U{{12..20}}, "
                                       f"edge factors U{{8..32}}, {n_q} queries (60% SSSP / 40% PPR restart 0.15 "
                                       f"tol 1e-6) in one hyt_batch_run",
                           "graphs": len(graphs), "queries": n_q,
                           "sssp_queries": sum(q["kind"] == "sssp" for q in queries),
                           "total_edges": int(sum(E_of)), "total_vertices": int(sum(V_of)), "seed": args.seed,
                           "scales": [s for s, _, _ in specs], "edge_factors": [e for _, e, _ in specs]},
                "queries_per_s": n_q * world / (ms / 1e3),
                "one_at_a_time": {"ms": single_ms, "queries_per_s": n_q / (single_ms / 1e3),
                                  "speedup_of_batch": single_ms / ms},
                "batch": {"supersteps": st["supersteps"], "kernel_launches": st["kernel_launches"],
                          "graph_launches": st["graph_launches"], "state_bytes": st["state_bytes"],
                          "algorithmic_bytes": st["algorithmic_bytes"],
                          "achieved_gbs": st["algorithmic_bytes"] / (ms / 1e3) / 1e9,
                          "tuning": tuning, "autotune_s": tune_s},
                "e2e": {"value": traversed / e2e_wall / 1e9, "unit": UNIT, "queries_per_s": n_q / e2e_wall,
                        "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": int(sum(V_of[q["graph"]] * 4 for q in queries)),
                        "ms_per_step": e2e_wall * 1e3},
                "roofline": {"bound": "hbm", "achieved": st["algorithmic_bytes"] / (ms / 1e3) / 1e9,
                             "peak": load_peaks()[0], "unit": "GB/s",
                             "frac": st["algorithmic_bytes"] / (ms / 1e3) / 1e9 / load_peaks()[0],
                             "traffic": None, "peak_kind": load_peaks()[1]},
                "cpu_baseline": cpu, "parity": parity, "clocks": clk, "gpu_launches": st["kernel_launches"]}
        line["config"]["vertex_order"] = args.vertex_order
        print(json.dumps(line), flush=True)
    for g in graphs:
        g.close()


def query_parity(specs, queries, results):
    """Query results (index -> host array) against the oracle on the same
    graphs, rebuilt by the oracle's generator: SSSP labels against Dijkstra
    (exact), personalized PageRank L1 against the FP64 restatement."""
    from oracle.bindings import Oracle

    from concurrent.futures import ThreadPoolExecutor

    o = Oracle()
    host = {}
    for i in results:
        gi = queries[i]["graph"]
        if gi not in host:
            sc, ef, gseed = specs[gi]
            host[gi] = o.rmat(sc, ef, gseed)

    def check(i):
        q, out = queries[i], results[i]
        off, cols, w = host[q["graph"]]
        if q["kind"] == "sssp":
            d = o.dijkstra(off, cols, w, q["source"])
            want = np.where(d == np.iinfo(np.uint64).max, 0xFFFFFFFF, d).astype(np.uint32)
            return "sssp", int(np.count_nonzero(out.view(np.uint32) != want))
        r, _, _, _ = o.ppr_f64(off, cols, q["source"], q["restart"], q["tolerance"])
        return "ppr", float(np.abs(out.view(np.float32).astype(np.float64) - r).sum())

    sssp_n = sssp_bad = ppr_n = 0
    worst_l1 = 0.0
    with ThreadPoolExecutor(max_workers=8) as ex:
        for kind, v in ex.map(check, list(results)):
            if kind == "sssp":
                sssp_n += 1
                sssp_bad += v
            else:
                ppr_n += 1
                worst_l1 = max(worst_l1, v)
    return {"queries_checked": len(results), "sssp_checked": sssp_n, "sssp_mismatches": sssp_bad,
            "ppr_checked": ppr_n, "ppr_max_l1_vs_fp64": worst_l1, "ppr_l1_tolerance": 1e-5,
            "ok": bool(sssp_bad == 0 and worst_l1 <= 1e-5)}


def batch_cpu_sample(hyt, specs, queries):
    """The reference's sssp_cpu on the first SSSP query of the two smallest
    graphs and the FP64 PPR restatement on the first PPR query of the same
    graphs (the reference has no PPR); queries/s extrapolated from the
    sample's mean time per query."""
    from oracle.bindings import Oracle, Reference

    order = sorted(range(len(specs)), key=lambda i: (specs[i][0], specs[i][1]))[:2]
    o = Oracle()
    ref = Reference() if Reference.available() else None
    t, n, kinds = 0.0, 0, set()
    for gi in order:
        sc, ef, gseed = specs[gi]
        c = hyt.rmat(sc, ef, gseed)
        for kind in ("sssp", "ppr"):
            q = next((q for q in queries if q["graph"] == gi and q["kind"] == kind), None)
            if q is None:
                continue
            t0 = time.perf_counter()
            if kind == "sssp" and ref is not None:
                ref.sssp_cpu(c.row_offsets, c.column_indices, c.weights.astype(np.float32), q["source"])
                kinds.add("reference")
            elif kind == "sssp":
                o.sssp(c.row_offsets, c.column_indices, c.weights.astype(np.float32), q["source"])
                kinds.add("port")
            else:
                o.ppr_f64(c.row_offsets, c.column_indices, q["source"])
                kinds.add("port")
            t += time.perf_counter() - t0
            n += 1
    if n == 0:
        return None
    return {"value": n / t, "unit": "queries/s", "cores": 1,
            "kind": "reference" if kinds == {"reference"} else "port",
            "sample": f"{n} queries on the two smallest graphs of the batch (reference sssp_cpu for SSSP, FP64 "
                      f"PPR restatement for PPR), {t:.2f} s"}


def run_serve_workload(args, rank, world, pg):
    """Served stream: 8 resident R-MAT graphs (scales 16-20, 22-24, edge
    factor 16); requests 70% SSSP / 30% PPR (restart 0.15, tol 1e-6) on a
    uniformly chosen graph from a source uniform over out-degree > 0;
    admission by a 16 GiB per-query-state budget.  Measures: capacity
    (every request submitted at once), open-loop Poisson sweeps (latency
    p50 / p99 and achieved queries/s per offered rate), and the same
    requests solved one at a time with hyt_sssp / hyt_ppr."""
    import threading
    import torch
    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    scales = [16, 17, 18, 19, 20, 22, 23, 24]
    graphs, pools = [], []
    gflags = capi.HYT_GRAPH_ALL | (capi.HYT_GRAPH_HUB_ORDER if args.vertex_order == "hub" else 0)
    for sc in scales:
        d = hyt.rmat(sc, 16, args.seed + sc, device=True)
        off = np.empty(d.num_vertices + 1, np.uint64)
        capi.copy(off.ctypes.data, C.cast(d.buffers.row_offsets, C.c_void_p).value, off.nbytes)
        graphs.append(hyt.Graph(d, flags=gflags))
        d.free()
        pools.append(hyt.pick_sources(off, args.seed + 7 * sc, 4096))
    V_of = [g.num_vertices for g in graphs]
    E_of = [g.num_edges for g in graphs]

    def make_requests(n, seed):
        r = np.random.default_rng(seed)
        gi = r.integers(0, len(graphs), n)
        kind = np.where(r.random(n) < 0.7, "sssp", "ppr")
        src = [int(pools[g][r.integers(0, len(pools[g]))]) for g in gi]
        return [(int(g), str(k), s) for g, k, s in zip(gi, kind, src)]

    # results land in a ring of 32 device buffers per (graph, kind): the
    # result copy stays on the path without one buffer per request
    ring = {(g, k): [torch.empty(V_of[g], dtype=torch.int32 if k == "sssp" else torch.float32, device="cuda")
                     for _ in range(32)] for g in range(len(graphs)) for k in ("sssp", "ppr")}
    ring_pos = {key: 0 for key in ring}

    def take_out(g, k):
        i = ring_pos[(g, k)]
        ring_pos[(g, k)] = (i + 1) % 32
        return ring[(g, k)][i]

    def serve(srv, reqs, rate):
        """Submits reqs open-loop at `rate` (None = all at once); returns
        (latencies ms, seconds from the first arrival to the last completion)."""
        lat, meta = [], {}
        gaps = np.random.default_rng(len(reqs)).exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
        arrivals = np.cumsum(gaps)
        t_start = time.perf_counter()

        def submitter():
            for (g, k, s), ta in zip(reqs, arrivals):
                now = time.perf_counter() - t_start
                if ta > now:
                    time.sleep(ta - now)
                t = srv.submit(g, k, s, out=take_out(g, k), restart=0.15, tolerance=1e-6)
                meta[t] = True

        th = threading.Thread(target=submitter)
        th.start()
        n_done, t_last = 0, t_start
        while n_done < len(reqs):
            for c in srv.poll(1024, wait_ms=5):
                if c["status"] != 0:
                    raise SystemExit(f"query failed with status {c['status']}")
                lat.append(c["latency_ms"])
                n_done += 1
                t_last = time.perf_counter()
        th.join()
        return np.array(lat), t_last - t_start

    with hyt.Server(graphs) as srv:
        serve(srv, make_requests(200, 1), None)  # warm-up
        reqs = make_requests(args.requests, 2)
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        lat, wall = serve(srv, reqs, None)
        clk = clocks.stop()
        cap_qps = len(reqs) / wall
        cap = {"requests": len(reqs), "wall_s": wall, "queries_per_s": cap_qps,
               "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}
        sweep = []
        for rate in [float(x) for x in args.rates.split(",") if x]:
            n = int(min(args.requests, max(50, rate * args.rate_seconds)))
            lat, wall = serve(srv, make_requests(n, int(rate)), rate)
            sweep.append({"offered_qps": rate, "requests": n, "achieved_qps": n / wall,
                          "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                          "mean_ms": float(lat.mean())})
        server_stats = srv.stats()
        # parity: one SSSP and one PPR per graph through the server, each into
        # its own buffer, checked against the oracle
        verify = [(gi, k, int(pools[gi][1 + (k == "ppr")])) for gi in range(len(graphs)) for k in ("sssp", "ppr")]
        vouts = [torch.empty(V_of[g], dtype=torch.int32 if k == "sssp" else torch.float32, device="cuda")
                 for g, k, _ in verify]
        vt = {srv.submit(g, k, x, out=o, restart=0.15, tolerance=1e-6): i
              for i, ((g, k, x), o) in enumerate(zip(verify, vouts))}
        vdone = 0
        while vdone < len(verify):
            vdone += len(srv.poll(64, wait_ms=50))
        torch.cuda.synchronize()
        vres = {i: vouts[i].cpu().numpy() for i in vt.values()}
    parity = None
    if rank == 0 and not args.no_parity:
        specs = [(sc, 16, args.seed + sc) for sc in scales]
        parity = query_parity(specs, [{"graph": g, "kind": k, "source": x, "restart": 0.15, "tolerance": 1e-6}
                                      for g, k, x in verify], vres)
    # one at a time: the same request mix, solved back to back, with every
    # graph's solver state allocated before timing
    sample = make_requests(min(400, args.requests), 3)
    for gi in range(len(graphs)):
        s0 = int(pools[gi][0])
        graphs[gi].sssp(s0, out=take_out(gi, "sssp"))
        graphs[gi].ppr(s0, out=take_out(gi, "ppr"))
    torch.cuda.synchronize()
    lat1 = []
    t0 = time.perf_counter()
    for g, k, s in sample:
        o = take_out(g, k)
        ts = time.perf_counter()
        (graphs[g].sssp(s, out=o) if k == "sssp" else graphs[g].ppr(s, out=o))
        lat1.append((time.perf_counter() - ts) * 1e3)
    single_qps = len(sample) / (time.perf_counter() - t0)
    for g in graphs:
        g.close()
    if rank == 0:
        line = {"metric": METRIC, "value": cap_qps * world, "unit": "queries/s", "n_gpus": world, "steps": 1,
                "warmup": 1, "ms_per_step": 1e3 * cap["wall_s"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (PPR) / u32 (SSSP)", "data": "synthetic",
                "config": {"workload": "served stream: 8 resident R-MAT graphs (scales 16,17,18,19,20,22,23,24, "
                                       "edge factor 16), 70% SSSP / 30% PPR (restart 0.15, tol 1e-6), uniform "
                                       "graph, source uniform over out-degree > 0, 16 GiB per-query-state budget, "
                                       "continuous batching",
                           "graphs_edges": E_of, "requests": args.requests, "seed": args.seed},
                "capacity": cap, "sweep": sweep,
                "one_at_a_time": {"requests": len(sample), "queries_per_s": single_qps,
                                  "p50_ms": float(np.percentile(lat1, 50)), "p99_ms": float(np.percentile(lat1, 99))},
                "speedup_vs_one_at_a_time": cap_qps / single_qps, "parity": parity,
                "server": server_stats, "clocks": clk, "gpu_launches": server_stats.get("graph_launches")}
        line["config"]["vertex_order"] = args.vertex_order
        print(json.dumps(line), flush=True)


def hubsort_config(args, V, E):
    return {"workload": f"hub sorting (HubSorter::sort, hub_fraction {args.hub_fraction}) + vertex reordering "
                        f"(CSRGraph::reorder_vertices) of R-MAT scale {args.scale} edge factor {args.edge_factor} "
                        f"with uint32 weights",
            "scale": args.scale, "edge_factor": args.edge_factor, "vertices": V, "edges": E,
            "hub_fraction": args.hub_fraction, "rmat_abc": [0.57, 0.19, 0.19], "seed": args.seed,
            "parallelism": f"replicas x{args.gpus}",
            "l2": "inputs larger than L2 (CSR + weights > 2 GB vs 126 MB L2)"}


def reference_hubsort(off, cols, w, fraction):
    """The reference's HubSorter::sort + CSRGraph::reorder_vertices (its own
    compiled code when available, else the oracle's restatement), one pass
    over the full graph.  Returns (seconds, kind)."""
    from oracle.bindings import Oracle, Reference

    if Reference.available():
        ref = Reference()
        t0 = time.perf_counter()
        order, _, _ = ref.hub_sort(off, cols, fraction)
        ref.reorder(off, cols, w.view(np.float32), order)
        return time.perf_counter() - t0, "reference"
    ora = Oracle()
    t0 = time.perf_counter()
    order, _, _ = ora.hub_sort(off, cols, fraction)
    ora.reorder(off, cols, w, order)
    return time.perf_counter() - t0, "port"


def run_hubsort_workload(args, rank, world, local, pg):
    """One step = hyt_hub_sort + hyt_csr_reorder of the device-resident graph
    (device in, device out).  Metric: edges hub-sorted and reordered per
    second."""
    import torch

    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    peak_gbs, peak_kind = load_peaks()
    d = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = d.num_vertices, d.num_edges
    order_d = torch.empty(V, dtype=torch.int32, device="cuda")
    scores_d = torch.empty(V, dtype=torch.float64, device="cuda")

    def step(collect):
        a, b = {}, {}
        hyt.hub_sort(d, args.hub_fraction, order_out=order_d, scores_out=scores_d, stats=a)
        r = hyt.reorder(d, order_d, device=True, stats=b)
        r.free()
        collect.append((a, b))

    warm = []
    for _ in range(args.warmup):
        step(warm)
    stream = torch.cuda.current_stream()
    clocks = ClockSampler(local)
    clocks.start()
    timed = []
    barrier(pg)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        step(timed)  # host-synchronous calls on the library's own stream
    ev1.record(stream)
    barrier(pg)
    wall_ms = 1e3 * (time.perf_counter() - t0)
    clk = clocks.stop()
    ms = max_over_ranks(pg, max(ev0.elapsed_time(ev1), wall_ms))
    value = replica_value(E * args.steps, world, ms) / 1e9
    hs_ms = sum(a["kernel_ms"] for a, _ in timed) / args.steps
    rp_ms = sum(b["kernel_ms"] for _, b in timed) / args.steps
    hs_bytes, rp_bytes = timed[0][0]["kernel_bytes"], timed[0][1]["kernel_bytes"]
    dev_ms = sum(a["device_ms"] + b["device_ms"] for a, b in timed) / args.steps
    alg_bytes = timed[0][0]["algorithmic_bytes"] + timed[0][1]["algorithmic_bytes"]
    if rp_ms >= hs_ms:
        kern, kb, kms = "permute_edges_kernel", rp_bytes, rp_ms
    else:
        kern, kb, kms = "degree_pass_kernel", hs_bytes, hs_ms
    roof = {"kernel": kern, "bound": "hbm", "achieved": kb / (kms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
            "frac": kb / (kms / 1e3) / 1e9 / peak_gbs, "traffic": None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": kb, "avg_launch_ms": kms,
            "other": {"degree_pass_kernel": {"ms": hs_ms, "bytes": hs_bytes},
                      "permute_edges_kernel": {"ms": rp_ms, "bytes": rp_bytes}},
            "whole_step_device_ms": dev_ms, "whole_step_algorithmic_bytes": alg_bytes,
            "whole_step_gbs": alg_bytes / (dev_ms / 1e3) / 1e9}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        tr = json.loads(traffic_file.read_text()).get(f"hubsort_s{args.scale}_ef{args.edge_factor}", {})
        roof["traffic"] = tr.get(kern)
        roof["traffic_measured"] = bool(tr.get("measured", False))
    launches = sum(a["kernel_launches"] + b["kernel_launches"] for a, b in timed)

    # effect on the solvers: PageRank + 8 SSSP sources on the original and on
    # the reordered graph (same results up to the renaming)
    effect = None
    if not args.no_effect:
        off_np = np.empty(V + 1, np.uint64)
        capi.copy(off_np.ctypes.data, C.cast(d.buffers.row_offsets, C.c_void_p).value, off_np.nbytes)
        srcs = [int(x) for x in hyt.pick_sources(off_np, args.seed, 8)]
        order_np = order_d.cpu().numpy().view(np.uint32)
        inv = np.empty_like(order_np)
        inv[order_np] = np.arange(V, dtype=np.uint32)
        r = hyt.reorder(d, order_d, device=True)
        effect = {}
        for name, g_csr, ss in (("original", d, srcs), ("hub_sorted", r, [int(inv[x]) for x in srcs])):
            with hyt.Graph(g_csr) as g:
                pr_out = torch.empty(V, dtype=torch.float32, device="cuda")
                di_out = torch.empty(V, dtype=torch.int32, device="cuda")
                g.pagerank(out=pr_out)
                prm = min(g.pagerank(out=pr_out)[1]["device_ms"] for _ in range(2))
                g.sssp(ss[0], out=di_out)
                sms = [g.sssp(x, out=di_out)[1]["device_ms"] for x in ss]
                effect[name] = {"pagerank_ms": prm, "sssp_ms_per_source": float(np.mean(sms))}
        r.free()
        effect["speedup"] = {k: effect["original"][k] / effect["hub_sorted"][k]
                             for k in ("pagerank_ms", "sssp_ms_per_source")}

    # e2e: the C ABI with pinned HOST buffers in and out
    off_t, cols_t, w_t = host_graph_from_device(d)
    d.free()
    del order_d, scores_d
    torch.cuda.empty_cache()
    csr = capi.hyt_csr()
    csr.num_vertices, csr.num_edges = V, E
    csr.row_offsets, csr.column_indices, csr.weights = off_t.data_ptr(), cols_t.data_ptr(), w_t.data_ptr()
    csr.weight_kind = capi.HYT_WEIGHTS_U32
    order_h = torch.empty(V, dtype=torch.int32, pin_memory=True)
    scores_h = torch.empty(V, dtype=torch.float64, pin_memory=True)

    def e2e_step():
        n = C.c_uint64()
        capi.check(capi.lib.hyt_hub_sort(C.byref(csr), args.hub_fraction, order_h.data_ptr(), scores_h.data_ptr(),
                                         C.byref(n), None))
        b = capi.hyt_csr_buffers()
        capi.check(capi.lib.hyt_csr_reorder(C.byref(csr), order_h.data_ptr(), 0, C.byref(b), None))
        capi.check(capi.lib.hyt_csr_buffers_free(C.byref(b)))

    e2e_step()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    barrier(pg)
    e2e_ms = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
    e2e_value = replica_value(E * args.e2e_steps, world, e2e_ms) / 1e9
    # hub sort: offsets + ids in, order + scores out; reorder: offsets, ids,
    # weights and order in, offsets, ids and weights out
    h2d = (V + 1) * 8 + E * 4 + (V + 1) * 8 + E * 8 + V * 4
    d2h = V * 12 + (V + 1) * 8 + E * 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, kind = reference_hubsort(off_t.numpy().view(np.uint64), cols_t.numpy().view(np.uint32),
                                    w_t.numpy().view(np.uint32), args.hub_fraction)
        cpu = {"value": E / t / 1e9, "unit": "Gedges/s", "cores": 1, "kind": kind,
               "sample": f"one HubSorter::sort + CSRGraph::reorder_vertices of the full graph, {t:.1f} s"}
    if rank == 0:
        line = {"metric": "hub sort + reorder throughput", "value": value, "unit": "Gedges/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64 (f64 scores)",
                "data": "synthetic", "config": hubsort_config(args, V, E),
                "e2e": {"value": e2e_value, "unit": "Gedges/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / args.e2e_steps,
                        "steps": args.e2e_steps},
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
                "effect_on_solvers": effect}
        print(json.dumps(line), flush=True)


def write_edge_text(path, src, dst, w=None, V=1):
    """Writes "source destination [weight]" lines with fixed-width decimal
    fields (leading zeros are plain decimal to the loader), vectorised."""
    nd = max(1, len(str(max(V - 1, 1))))
    nw = 0 if w is None else max(1, len(str(int(w.max()) if w.size else 1)))

    def digits(x, n):
        out = np.empty((x.shape[0], n), np.uint8)
        y = x.astype(np.uint64)
        for k in range(n - 1, -1, -1):
            out[:, k] = (y % 10).astype(np.uint8) + 48
            y //= 10
        return out

    with open(path, "wb") as f:
        f.write(b"# R-MAT edge list: source destination" + (b" weight" if w is not None else b"") + b"\n")
        step = 1 << 22
        for b in range(0, src.shape[0], step):
            e = min(b + step, src.shape[0])
            n = e - b
            parts = [digits(src[b:e], nd), np.full((n, 1), 32, np.uint8), digits(dst[b:e], nd)]
            if w is not None:
                parts += [np.full((n, 1), 32, np.uint8), digits(w[b:e], nw)]
            parts.append(np.full((n, 1), 10, np.uint8))
            f.write(np.concatenate(parts, axis=1).tobytes())


def pinned_h2d_gbs():
    """Best pinned host->device copy bandwidth of 256 MiB (GB/s)."""
    import torch

    h = torch.empty(256 << 20, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d.copy_(h, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, (256 << 20) / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def load_config(args, V, E, Vt, Et):
    return {"workload": f"GraphLoader::load_edge_list of an R-MAT scale {args.text_scale} edge factor "
                        f"{args.edge_factor} text edge list with uint weights (file -> CSR in HBM), and the binary "
                        f"CSR file of R-MAT scale {args.scale} (file -> CSR in HBM), page cache warm",
            "text_scale": args.text_scale, "text_vertices": Vt, "text_edges": Et, "binary_scale": args.scale,
            "binary_vertices": V, "binary_edges": E, "edge_factor": args.edge_factor, "seed": args.seed,
            "parallelism": f"replicas x{args.gpus}"}


def run_load_workload(args, rank, world, local, pg):
    """One step = hyt_load_edge_list of the text file to the device + the
    CSR construction; the binary file's device load is timed beside it."""
    import shutil
    import tempfile

    import torch

    import hytgraph_b200 as hyt

    peak_gbs, peak_kind = load_peaks()
    tmp = tempfile.mkdtemp(prefix="hyt_load_")
    try:
        # text edge list, records in CSR order
        t = hyt.rmat(args.text_scale, args.edge_factor, args.seed)
        Vt, Et = t.num_vertices, t.num_edges
        src = np.repeat(np.arange(Vt, dtype=np.uint32), np.diff(t.row_offsets).astype(np.int64))
        text_path = os.path.join(tmp, "g.el")
        write_edge_text(text_path, src, t.column_indices, t.weights, Vt)
        text_bytes = os.path.getsize(text_path)
        sample_path = os.path.join(tmp, "sample.el")
        ns = min(Et, 1 << 21)
        write_edge_text(sample_path, src[:ns], t.column_indices[:ns], t.weights[:ns], Vt)
        del t, src
        # binary file of the larger graph
        d = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
        V, E = d.num_vertices, d.num_edges
        bin_path = os.path.join(tmp, "g.csr")
        hyt.save_csr(d, bin_path)
        d.free()
        bin_bytes = os.path.getsize(bin_path)

        def step(collect):
            st = {}
            g = hyt.load_edge_list(text_path, Vt, True, device=True, stats=st)
            g.free()
            collect.append(st)

        warm = []
        for _ in range(args.warmup):
            step(warm)
        clocks = ClockSampler(local)
        clocks.start()
        timed = []
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step(timed)
        barrier(pg)
        ms = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
        clk = clocks.stop()
        value = replica_value(Et * args.steps, world, ms) / 1e9
        kms = sum(x["kernel_ms"] for x in timed) / args.steps
        kb = timed[0]["kernel_bytes"]
        roof = {"kernel": "CSR construction (pack + radix sort + offsets + unpack)", "bound": "hbm",
                "achieved": kb / (kms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
                "frac": kb / (kms / 1e3) / 1e9 / peak_gbs, "traffic": None, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": kb, "avg_launch_ms": kms,
                "note": "algorithmic bytes = edges read and written once + offsets; the radix sort's passes "
                        "are the overhead"}
        parse_ms = sum(x["read_ms"] for x in timed) / args.steps
        # binary file -> device
        link = pinned_h2d_gbs()
        bl = []
        for i in range(args.warmup + args.steps):
            st = {}
            g = hyt.load_csr(bin_path, device=True, stats=st)
            g.free()
            if i >= args.warmup:
                bl.append(st)
        b_ms = sum(x["total_ms"] for x in bl) / len(bl)
        binary = {"file_bytes": bin_bytes, "ms_per_load": b_ms, "gbs": bin_bytes / (b_ms / 1e3) / 1e9,
                  "pinned_h2d_gbs": link, "frac_of_h2d": bin_bytes / (b_ms / 1e3) / 1e9 / link,
                  "read_threads": bl[0]["threads"], "check_ms": sum(x["kernel_ms"] for x in bl) / len(bl),
                  "edges_per_s": E / (b_ms / 1e3)}
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            tc, kind = reference_load(sample_path, Vt)
            cpu = {"value": ns / tc / 1e9, "unit": "Gedges/s", "cores": 1, "kind": kind,
                   "sample": f"GraphLoader::load_edge_list of the first {ns} edges of the same file, {tc:.1f} s"}
        if rank == 0:
            line = {"metric": "edge-list load throughput (file -> CSR in HBM)", "value": value, "unit": "Gedges/s",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "u32 ids, f32 weights", "data": "synthetic", "config": load_config(args, V, E, Vt, Et),
                    "e2e": {"value": value, "unit": "Gedges/s", "h2d_bytes_per_step": Et * 12,
                            "d2h_bytes_per_step": 0, "note": "the step is already host file -> device CSR"},
                    "text": {"file_bytes": text_bytes, "parse_ms": parse_ms,
                             "parse_gbs": text_bytes / (parse_ms / 1e3) / 1e9, "threads": timed[0]["threads"],
                             "device_ms": sum(x["device_ms"] for x in timed) / args.steps},
                    "binary": binary, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                    "gpu_launches": 5 * args.steps}
            print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def reference_load(path, V):
    """The reference's GraphLoader::load_edge_list (its own compiled code when
    available, else the oracle's restatement) on `path`: (seconds, kind)."""
    from oracle.bindings import Oracle, Reference

    if Reference.available():
        t0 = time.perf_counter()
        Reference().load_edge_list(path, V, True)
        return time.perf_counter() - t0, "reference"
    t0 = time.perf_counter()
    Oracle().load_edge_list(path, V, True)
    return time.perf_counter() - t0, "port"


def run_contrib_workload(args, rank, world, local, pg):
    """One step = pagerank_contributions of every vertex (mid-solve ranks),
    ContributionScheduler::schedule of all V vertices by contribution, and
    the per-partition priorities (2^20-vertex partitions)."""
    import torch

    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    peak_gbs, peak_kind = load_peaks()
    d = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = d.num_vertices, d.num_edges
    off_np = np.empty(V + 1, np.uint64)
    capi.copy(off_np.ctypes.data, C.cast(d.buffers.row_offsets, C.c_void_p).value, off_np.nbytes)
    g = hyt.Graph(d)
    ranks = torch.empty(V, dtype=torch.float32, device="cuda")
    g.pagerank(max_iterations=3, tolerance=1e-30, out=ranks)
    contrib = torch.empty(V, dtype=torch.float64, device="cuda")
    items = torch.arange(V, dtype=torch.int64, device="cuda")
    ordered = torch.empty(V, dtype=torch.int64, device="cuda")
    P = max(1, (V + args.partition_vertices - 1) // args.partition_vertices)
    bounds = torch.tensor([min(i * args.partition_vertices, V) for i in range(P + 1)], dtype=torch.int64,
                          device="cuda")
    prio = torch.empty(P, dtype=torch.float64, device="cuda")

    def step(collect):
        t0 = time.perf_counter()
        g.pagerank_contributions(ranks, 0.85, out=contrib)
        t1 = time.perf_counter()
        _, m = hyt.contribution_schedule(items, contrib, out=ordered)
        t2 = time.perf_counter()
        hyt.partition_contributions(contrib, bounds, out=prio)
        t3 = time.perf_counter()
        collect.append((1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2), m))

    warm = []
    for _ in range(args.warmup):
        step(warm)
    clocks = ClockSampler(local)
    clocks.start()
    timed = []
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(timed)
    barrier(pg)
    ms = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
    clk = clocks.stop()
    value = replica_value(V * args.steps, world, ms) / 1e9
    c_ms = sum(x[0] for x in timed) / args.steps
    s_ms = sum(x[1] for x in timed) / args.steps
    p_ms = sum(x[2] for x in timed) / args.steps
    kb = 12 * E + 20 * V  # source id, rank and degree gathers per in-edge; offsets, rank, output per vertex
    roof = {"kernel": "pagerank_contrib_kernel (+ dangling partials)", "bound": "hbm",
            "achieved": kb / (c_ms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
            "frac": kb / (c_ms / 1e3) / 1e9 / peak_gbs, "traffic": None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": kb, "avg_launch_ms": c_ms,
            "note": "launch time from the host clock around the synchronous call"}
    # e2e: host arrays in and out through the C ABI
    ranks_h = ranks.cpu().numpy()
    t0 = time.perf_counter()
    ch = g.pagerank_contributions(ranks_h, 0.85)
    oh, _ = hyt.contribution_schedule(np.arange(V, dtype=np.uint64), ch)
    e2e_ms = 1e3 * (time.perf_counter() - t0)
    g.close()
    d.free()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.bindings import Reference

        host = hyt.rmat(args.scale, args.edge_factor, args.seed) if args.scale <= 20 else None
        if host is None:
            dd = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
            off_t, cols_t, _ = host_graph_from_device(dd)
            dd.free()
            hoff, hcols = off_t.numpy().view(np.uint64), cols_t.numpy().view(np.uint32)
        else:
            hoff, hcols = host.row_offsets, host.column_indices
        if Reference.available():
            ref = Reference()
            tt = time.perf_counter()
            rc = ref.pagerank_contributions(hoff, hcols, ranks_h, 0.85)
            ref.contribution_schedule(np.arange(V, dtype=np.uint64), rc)
            tc = time.perf_counter() - tt
            cpu = {"value": V / tc / 1e9, "unit": "Gvertices/s", "cores": 1, "kind": "reference",
                   "sample": f"one pagerank_contributions + ContributionScheduler::schedule of all V on the full "
                             f"graph, {tc:.1f} s"}
    if rank == 0:
        line = {"metric": "contribution pass + schedule throughput", "value": value, "unit": "Gvertices/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 contributions",
                "data": "synthetic",
                "config": {"workload": f"pagerank_contributions (ranks after 3 iterations) + schedule of every "
                                       f"vertex + priorities of {P} partitions, R-MAT scale {args.scale} edge "
                                       f"factor {args.edge_factor}",
                           "vertices": V, "edges": E, "partitions": P, "seed": args.seed,
                           "parallelism": f"replicas x{args.gpus}"},
                "e2e": {"value": V / (e2e_ms / 1e3) / 1e9, "unit": "Gvertices/s", "h2d_bytes_per_step": V * 12,
                        "d2h_bytes_per_step": V * 16, "ms_per_step": e2e_ms},
                "phases_ms": {"pagerank_contributions": c_ms, "schedule": s_ms, "partition_priorities": p_ms},
                "schedule_metrics": timed[0][3], "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": 10 * args.steps}
        print(json.dumps(line), flush=True)


def run_ppr8_workload(args, rank, world, local, pg):
    """One step = 8 personalized PageRank queries (restart 0.15, tol 1e-6)
    from seeded sources, packed into one hyt_ppr_multi call; the same 8
    queries through hyt_ppr one at a time are timed beside it.  The line
    also reports 8 SSSP sources in one hyt_sssp_multi solve against the
    same sources through hyt_sssp (device time, labels compared)."""
    import torch

    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    peak_gbs, peak_kind = load_peaks()
    d = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = d.num_vertices, d.num_edges
    off_np = np.empty(V + 1, np.uint64)
    capi.copy(off_np.ctypes.data, C.cast(d.buffers.row_offsets, C.c_void_p).value, off_np.nbytes)
    gflags = capi.HYT_GRAPH_ALL | (capi.HYT_GRAPH_HUB_ORDER if args.vertex_order == "hub" else 0)
    g = hyt.Graph(d, flags=gflags)
    d.free()
    out = torch.empty((8, V), dtype=torch.float32, device="cuda")
    one = torch.empty(V, dtype=torch.float32, device="cuda")
    step_no = [0]

    def sources():
        step_no[0] += 1
        return np.array(hyt.pick_sources(off_np, args.seed + step_no[0], 8), np.uint32)

    def step(collect):
        _, st = g.ppr_multi(sources(), out=out)
        collect.append(st)

    warm = []
    for _ in range(args.warmup):
        step(warm)
    clocks = ClockSampler(local)
    clocks.start()
    timed = []
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(timed)
    barrier(pg)
    ms = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
    clk = clocks.stop()
    value = replica_value(8 * args.steps, world, ms)
    # one at a time: the same kind of queries through hyt_ppr
    g.ppr(int(sources()[0]), out=one)
    t1 = time.perf_counter()
    singles = []
    for s in sources():
        _, st = g.ppr(int(s), out=one)
        singles.append(st)
    single_ms = 1e3 * (time.perf_counter() - t1)
    dev_ms = sum(x[0]["device_ms"] for x in timed) / args.steps
    iters = sum(max(y["iterations"] for y in x) for x in timed) / args.steps
    kb = timed[0][0]["algorithmic_bytes"] / max(max(y["iterations"] for y in timed[0]), 1)
    it_ms = dev_ms / max(iters, 1)
    # 8 SSSP sources in one hyt_sssp_multi solve against the same sources
    # one at a time (hyt_sssp): labels identical, timed on the device
    ss_out = torch.empty((8, V), dtype=torch.int32, device="cuda")
    ss_one = torch.empty(V, dtype=torch.int32, device="cuda")
    src8 = sources()
    g.sssp_multi(src8, out=ss_out)
    torch.cuda.synchronize()
    ms_multi, ms_single, multi_st = [], [], None
    for _ in range(max(args.steps, 1)):
        src8 = sources()
        _, multi_st = g.sssp_multi(src8, out=ss_out)
        ms_multi.append(multi_st["device_ms"])
        tot = 0.0
        for lane, s_ in enumerate(src8):
            _, st1 = g.sssp(int(s_), out=ss_one)
            tot += st1["device_ms"]
            if lane == 0:
                torch.cuda.synchronize()
                same = bool(torch.equal(ss_one, ss_out[0]))
                if not same:
                    raise SystemExit("hyt_sssp_multi lane 0 differs from hyt_sssp")
        ms_single.append(tot)
    sssp8 = {"sources_per_solve": 8, "ms_per_solve": statistics.median(ms_multi),
             "one_at_a_time_ms_for_8": statistics.median(ms_single),
             "speedup_vs_one_at_a_time": statistics.median(ms_single) / statistics.median(ms_multi),
             "rounds": multi_st["iterations"], "relaxations_per_edge": multi_st["edges_processed"] / E,
             "gteps": 8 * E / (statistics.median(ms_multi) / 1e3) / 1e9}
    roof = {"kernel": "ppr8 iteration (prep + rows + long rows)", "bound": "hbm",
            "achieved": kb / (it_ms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
            "frac": kb / (it_ms / 1e3) / 1e9 / peak_gbs, "traffic": None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": kb, "avg_launch_ms": it_ms,
            "note": "per iteration of the packed solve: 36 B per in-edge (id + a 32-byte sector of the 8 "
                    "queries' contributions) + 108 B per vertex"}
    g.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.bindings import Oracle

        host = hyt.rmat(min(args.scale, 20), args.edge_factor, args.seed)
        src = int(hyt.pick_sources(host.row_offsets, args.seed, 1)[0])
        tt = time.perf_counter()
        Oracle().ppr_f64(host.row_offsets, host.column_indices, src, 0.15, 1e-6, 100)
        tc = time.perf_counter() - tt
        cpu = {"value": 1.0 / tc * (host.num_edges / E), "unit": "queries/s (scaled to this graph's edges)",
               "cores": 1, "kind": "port",
               "sample": f"one FP64 personalized PageRank (the oracle's restatement; the reference has no PPR) on "
                         f"R-MAT scale {min(args.scale, 20)}, {tc:.1f} s, scaled by the edge ratio"}
    if rank == 0:
        line = {"metric": "personalized PageRank queries/s (8 packed per solve)", "value": value,
                "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 values, f64 sums", "data": "synthetic",
                "config": {"workload": f"8 PPR queries (restart 0.15, tol 1e-6) per step on R-MAT scale {args.scale} "
                                       f"edge factor {args.edge_factor}, sources seeded per step",
                           "vertices": V, "edges": E, "vertex_order": args.vertex_order, "seed": args.seed,
                           "parallelism": f"replicas x{args.gpus}"},
                "one_at_a_time": {"queries_per_s": 8 / (single_ms / 1e3), "ms_per_query": single_ms / 8,
                                  "iterations": [s_["iterations"] for s_ in singles]},
                "speedup_vs_one_at_a_time": value / (8 / (single_ms / 1e3)),
                "packed": {"device_ms_per_solve": dev_ms, "iterations_per_solve": iters}, "sssp8": sssp8,
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": None}
        print(json.dumps(line), flush=True)


def run_shard_workload(args, rank, world, local, pg):
    """The inhbm step (PageRank to L1 <= 1e-6 + SSSP from the seeded
    sources) on ONE graph split by vertex range over all ranks
    (hytgraph_b200.ShardedGraph): every rank builds the same graph, computes
    its range, and the vectors move over NCCL between iterations / rounds.
    Strong scaling: the total work is fixed as ranks are added."""
    import torch

    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    peak_gbs, peak_kind = load_peaks()
    stream = torch.cuda.current_stream()
    d = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = d.num_vertices, d.num_edges
    off_h, cols_h, w_h = host_graph_from_device(d)
    off_np = off_h.numpy().view(np.uint64)
    sources = [int(x) for x in hyt.pick_sources(off_np, args.seed, args.sources)]
    gflags = capi.HYT_GRAPH_ALL | (capi.HYT_GRAPH_HUB_ORDER if args.vertex_order == "hub" else 0)
    g = hyt.Graph(d, flags=gflags)
    d.free()
    sg = hyt.ShardedGraph(g)
    ranks_out = torch.empty(V, dtype=torch.float32, device="cuda")
    dist_out = torch.empty(V, dtype=torch.int32, device="cuda")

    def step(collect):
        _, st = sg.pagerank(out=ranks_out)
        collect["pr"].append(st)
        for s_ in sources:
            _, ss = sg.sssp(s_, out=dist_out)
            collect["sssp"].append(ss)

    warm = {"pr": [], "sssp": []}
    for _ in range(args.warmup):
        step(warm)
    clocks = ClockSampler(local)
    clocks.start()
    timed = {"pr": [], "sssp": []}
    barrier(pg)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(timed)
    ev1.record(stream)
    barrier(pg)
    clk = clocks.stop()
    ms = max_over_ranks(pg, ev0.elapsed_time(ev1))
    pr_it = sum(x["iterations"] for x in timed["pr"])
    rounds = sum(x["iterations"] for x in timed["sssp"])
    value = (E * pr_it + E * len(timed["sssp"])) / (ms / 1e3) / 1e9
    pr_ms = sum(x["ms"] for x in timed["pr"])
    ss_ms = sum(x["ms"] for x in timed["sssp"])
    pull, push = sg.kernels.info(capi.HYT_SHARD_PULL), sg.kernels.info(capi.HYT_SHARD_PUSH)
    it_bytes = 8 * E + 20 * V  # one PageRank iteration over the whole graph (as hyt_pagerank counts it)
    it_ms = pr_ms / max(pr_it, 1)
    roof = {"kernel": "shard_pr_step_kernel + slice broadcasts", "bound": "hbm",
            "achieved": it_bytes / (it_ms / 1e3) / 1e9, "peak": peak_gbs * world, "unit": "GB/s",
            "frac": it_bytes / (it_ms / 1e3) / 1e9 / (peak_gbs * world), "traffic": None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": it_bytes, "avg_launch_ms": it_ms,
            "note": "per PageRank iteration of the whole graph (all ranks' steps + the exchange, host-timed); "
                    "peak = measured HBM copy bandwidth x ranks"}
    # PageRank: init + one step per iteration + emit; SSSP: init + (collect, expand, sweep) per round + labels
    launches = sum(2 + x["iterations"] for x in timed["pr"]) + sum(3 + 3 * x["iterations"] for x in timed["sssp"])
    sg.close()
    g.close()

    # e2e: host CSR in, graph built and split, results back on the host
    csr_h = hyt.CSR(off_np, cols_h.numpy().view(np.uint32), w_h.numpy().view(np.uint32))

    def e2e_step():
        with hyt.Graph(csr_h, flags=gflags) as g2, hyt.ShardedGraph(g2) as sg2:
            _, st = sg2.pagerank()
            for s_ in sources:
                sg2.sssp(s_)
        return st["iterations"]

    e2e_step()
    barrier(pg)
    t0 = time.perf_counter()
    e2e_it = 0
    for _ in range(args.e2e_steps):
        e2e_it += e2e_step()
    barrier(pg)
    e2e_ms = max_over_ranks(pg, 1e3 * (time.perf_counter() - t0))
    e2e_value = (E * e2e_it + E * len(sources) * args.e2e_steps) / (e2e_ms / 1e3) / 1e9
    if rank == 0:
        line = {"metric": SHARD_METRIC, "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32 (PageRank) / u32 (SSSP)", "data": "synthetic",
                "config": shard_config(args, V, E, world),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": (V + 1) * 8 + 8 * E,
                        "d2h_bytes_per_step": 4 * V * (1 + len(sources)), "ms_per_step": e2e_ms / args.e2e_steps,
                        "steps": args.e2e_steps},
                "roofline": roof, "cpu_baseline": None, "clocks": clk, "gpu_launches": launches,
                "pagerank": {"iterations_per_solve": pr_it / args.steps, "ms_per_solve": pr_ms / args.steps,
                             "exchanged_bytes_per_solve": timed["pr"][0]["exchanged_bytes"]},
                "sssp": {"solves": len(timed["sssp"]), "ms_per_solve": ss_ms / len(timed["sssp"]),
                         "rounds_per_solve": rounds / len(timed["sssp"]),
                         "relaxations_per_edge_rank0_last_solve": push["edges_relaxed"] / E},
                "rank0_shard": {"pull_vertices": pull["vertex_end"] - pull["vertex_begin"],
                                "pull_edges": pull["edges"], "push_vertices": push["vertex_end"] - push["vertex_begin"],
                                "push_edges": push["edges"]}}
        print(json.dumps(line), flush=True)


SHARD_METRIC = "PR/SSSP GTEPS on one graph split over the ranks"


def shard_config(args, V, E, world):
    return dict(workload_config(args, V, E), parallelism=f"vertex-range shards x{world} (NCCL)",
                workload=f"one R-MAT scale {args.scale} edge factor {args.edge_factor} graph split by vertex "
                         f"range: PageRank to L1<=1e-6 + SSSP from {args.sources} seeded sources")


def workload_config(args, V, E):
    return {"workload": f"in-HBM R-MAT scale {args.scale} edge factor {args.edge_factor}: PageRank to L1<=1e-6 "
                        f"+ SSSP from {args.sources} seeded sources",
            "scale": args.scale, "edge_factor": args.edge_factor, "vertices": V, "edges": E,
            "sources": args.sources, "rmat_abc": [0.57, 0.19, 0.19], "weights": "uint32 uniform [1,63]",
            "seed": args.seed, "parallelism": f"replicas x{args.gpus}",
            "vertex_order": ("hub: stored in the reference's HubSorter order (built at graph creation, inside the "
                             "e2e step); sources and results in input ids") if args.vertex_order == "hub" else "input",
            "l2": "inputs larger than L2 (CSR + CSC + weights > 4 GB vs 126 MB L2)"}


def main():
    args = parse_args()
    import torch

    rank, world, local, pg = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference_arm(args, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    if args.workload == "hybrid":
        run_hybrid(args, rank, world, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "serve":
        run_serve_workload(args, rank, world, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "batch":
        run_batch_workload(args, rank, world, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "ppr8":
        run_ppr8_workload(args, rank, world, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "contrib":
        run_contrib_workload(args, rank, world, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "load":
        run_load_workload(args, rank, world, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "shard":
        run_shard_workload(args, rank, world, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "hubsort":
        run_hubsort_workload(args, rank, world, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    import hytgraph_b200 as hyt
    from hytgraph_b200 import capi

    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    peak_gbs, peak_kind = load_peaks()

    # ---- setup (untimed): generate on the GPU, build the resident graph ----
    dcsr = hyt.rmat(args.scale, args.edge_factor, args.seed, device=True)
    V, E = dcsr.num_vertices, dcsr.num_edges
    off_h, cols_h, w_h = host_graph_from_device(dcsr)
    off_np = off_h.numpy().view(np.uint64)
    sources = [int(s) for s in hyt.pick_sources(off_np, args.seed, args.sources)]
    gflags = capi.HYT_GRAPH_ALL | (capi.HYT_GRAPH_HUB_ORDER if args.vertex_order == "hub" else 0)
    graph = hyt.Graph(dcsr, stream=sptr, flags=gflags)
    dcsr.free()
    ranks_out = torch.empty(V, dtype=torch.float32, device="cuda")
    # one label array per source, so the timed run's results are all checked
    dist_outs = [torch.empty(V, dtype=torch.int32, device="cuda") for _ in sources]

    def step(collect):
        _, st = graph.pagerank(out=ranks_out, stream=sptr)
        collect["pr"].append(st)
        for s, d in zip(sources, dist_outs):
            _, ss = graph.sssp(s, out=d, stream=sptr)
            collect["sssp"].append(ss)

    warm = {"pr": [], "sssp": []}
    for _ in range(args.warmup):
        step(warm)

    # ---- timed region: device-resident inputs ----
    clocks = ClockSampler(local)
    clocks.start()
    timed = {"pr": [], "sssp": []}
    barrier(pg)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(timed)
    ev1.record(stream)
    barrier(pg)
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    ms = max_over_ranks(pg, ms_local)
    pr_it = sum(s["iterations"] for s in timed["pr"])
    traversed = E * pr_it + E * len(timed["sssp"])
    value = replica_value(traversed, world, ms) / 1e9

    # roofline: dominant kernel of the step (PageRank iteration vs SSSP rounds)
    pr_ms = sum(s["device_ms"] for s in timed["pr"])
    ss_ms = sum(s["device_ms"] for s in timed["sssp"])
    pr_bytes = sum(s["algorithmic_bytes"] for s in timed["pr"])
    ss_bytes = sum(s["algorithmic_bytes"] for s in timed["sssp"])
    pr_launch_ms = pr_ms / max(pr_it, 1)  # whole solve / iterations: includes init + loop overhead
    pr_gbs = (pr_bytes / max(pr_it, 1)) / (pr_launch_ms / 1e3) / 1e9
    ss_gbs = ss_bytes / (ss_ms / 1e3) / 1e9
    # pure kernel time of one PageRank iteration (per-launch events), same inputs
    _, prof = graph.pagerank(out=ranks_out, stream=sptr, flags=capi.HYT_RUN_PROFILE)
    kern_ms = prof["kernel_ms"] / max(prof["kernel_launches"], 1)
    staged = os.environ.get("HYT_STAGED") == "1"  # bulk-staged kernels are opt-in
    pr_name = "pr_staged_kernel+pr_reduce_kernel" if staged else "pr_iterate_kernel+pr_reduce_kernel"
    ss_name = ("sssp_pull_staged_kernel" if staged else "sssp_pull_kernel") + "+sssp_expand_kernel+sssp_hub_kernel"
    dominant = pr_name if pr_ms >= ss_ms else ss_name
    if dominant == pr_name:
        roof = {"kernel": dominant, "bound": "hbm", "achieved": pr_gbs, "peak": peak_gbs, "unit": "GB/s",
                "frac": pr_gbs / peak_gbs, "traffic": None, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": pr_bytes / max(pr_it, 1), "avg_launch_ms": pr_launch_ms,
                "kernel_only_launch_ms": kern_ms,
                "kernel_only_frac": (pr_bytes / max(pr_it, 1)) / (kern_ms / 1e3) / 1e9 / peak_gbs}
    else:
        roof = {"kernel": dominant, "bound": "hbm", "achieved": ss_gbs, "peak": peak_gbs, "unit": "GB/s",
                "frac": ss_gbs / peak_gbs, "traffic": None, "peak_kind": peak_kind,
                "launch": "one SSSP solve (all rounds of one source)",
                "algorithmic_bytes_per_launch": ss_bytes / max(len(timed["sssp"]), 1),
                "avg_launch_ms": ss_ms / max(len(timed["sssp"]), 1)}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        tr = json.loads(traffic_file.read_text()).get(f"s{args.scale}_ef{args.edge_factor}", {})
        roof["traffic"] = tr.get("pr_iteration" if dominant == pr_name else "sssp_solve")
        roof["traffic_measured"] = bool(tr.get("measured", False))

    launches = sum(s["total_launches"] for s in timed["pr"]) + sum(s["total_launches"] for s in timed["sssp"])
    # results of the timed run, for the parity check after the timed regions
    torch.cuda.synchronize()
    ranks_timed = ranks_out.cpu().numpy()
    dists_timed = [d.cpu().numpy().view(np.uint32) for d in dist_outs]
    del dist_outs

    # ---- e2e: the C-ABI with HOST (pinned) buffers, copies inside the timed region ----
    ranks_h = torch.empty(V, dtype=torch.float32, pin_memory=True)
    dist_h = torch.empty(V, dtype=torch.int32, pin_memory=True)
    csr_h = hyt.CSR(off_np, cols_h.numpy().view(np.uint32), w_h.numpy().view(np.uint32))
    graph.close()
    torch.cuda.empty_cache()

    def e2e_step():
        with hyt.Graph(csr_h, stream=sptr, flags=gflags) as g2:
            _, st = g2.pagerank(out=ranks_h, stream=sptr)
            its = st["iterations"]
            for s in sources:
                g2.sssp(s, out=dist_h, stream=sptr)
        return its

    e2e_step()
    barrier(pg)
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_it = 0
    for _ in range(args.e2e_steps):
        e2e_it += e2e_step()
    e1.record(stream)
    barrier(pg)
    e2e_wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(pg, max(e0.elapsed_time(e1), 1e3 * e2e_wall))
    e2e_value = (E * e2e_it + E * len(sources) * args.e2e_steps) * world / (e2e_ms / 1e3) / 1e9
    h2d = (V + 1) * 8 + E * 4 + E * 4
    d2h = V * 4 * (1 + len(sources))

    # ---- parity of the timed run against the oracle (rank 0) ----
    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_inhbm(off_np, csr_h.column_indices, csr_h.weights, sources, ranks_timed, dists_timed)
        parity["gpu_pr_iterations"] = int(timed["pr"][-1]["iterations"])

    # ---- CPU baseline (rank 0, N=1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        solvers = CpuSolvers()
        n_pr = parity["_ref_iterations"] if parity else 100
        n_ss = parity["_ref_rounds_source0"] if parity else 10
        t_step, parts, t_sample = cpu_baseline_sample(solvers, off_np, csr_h.column_indices,
                                                      csr_h.weights.astype(np.float32), sources[0], n_pr, n_ss,
                                                      len(sources))
        cpu = {"value": (E * n_pr + E * len(sources)) / t_step / 1e9, "unit": UNIT, "cores": solvers.cores,
               "kind": solvers.kind,
               "sample": (f"pagerank_cpu for 1 and 3 iterations and sssp_cpu for 1 and 3 rounds on this graph "
                          f"({t_sample:.1f} s); projected to one step (PageRank to convergence in the reference's "
                          f"{n_pr} iterations + {len(sources)} full SSSP solves of {n_ss} rounds), E counted per "
                          f"PageRank iteration and per SSSP source as above"),
               "projected_step_s": t_step, "parts": parts}
    if parity:
        parity.pop("_ref_iterations", None)
        parity.pop("_ref_rounds_source0", None)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (PageRank) / u32 (SSSP)",
                "data": "synthetic", "config": workload_config(args, V, E),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_ms / args.e2e_steps, "steps": args.e2e_steps},
                "roofline": roof, "cpu_baseline": cpu, "parity": parity, "clocks": clk, "gpu_launches": launches,
                "pagerank": {"iterations_per_solve": pr_it / args.steps, "ms_per_solve": pr_ms / args.steps,
                             "gteps": E * pr_it / (pr_ms / 1e3) / 1e9, "achieved_gbs": pr_gbs},
                "sssp": {"solves": len(timed["sssp"]), "ms_per_solve": ss_ms / len(timed["sssp"]),
                         "gteps": E * len(timed["sssp"]) / (ss_ms / 1e3) / 1e9,
                         "rounds_per_solve": sum(s["iterations"] for s in timed["sssp"]) / len(timed["sssp"]),
                         "relaxations_per_edge": sum(s["edges_processed"] for s in timed["sssp"]) / (
                             E * len(timed["sssp"])),
                         "achieved_gbs": ss_gbs}}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
