"""Vertex-range sharding over several GPUs: one process per GPU, each holding
the same graph and computing one contiguous range of internal vertex ids
(the hyt_shard_* entry points of include/hyt/capi.h), with the whole-graph
vectors exchanged through torch.distributed (NCCL over NVLink / NVSwitch on
a B200 node).

PageRank / personalized PageRank, per iteration: every process runs the
pull step over its rows; one all-gather of the owners' slices of the new
contribution vector (padded to the longest slice; 4 bytes per vertex of
payload) gives every process the whole vector; one all-reduce sums the
(L1 change, dangling mass) pair, so every process takes the same stop
decision as the single-GPU solver (residual <= tolerance, or the iteration
cap).

SSSP, per round: every process collects its improved vertices and one
all-reduce sums their out-edges; when that frontier is dense (more than
E / 4 out-edges, the single-GPU rule) every process sweeps its rows over
the CSC (pull), else it pushes its frontier's out-edges into its copy of
the key vector (label XOR 0x80000000 as int32).  One MIN all-reduce over
V + 1 words then merges the copies and the idle flags; the solve ends in
the first round in which no shard had a frontier.  Labels are
bit-identical to the single-GPU solver.

The kernels sit behind a small interface (``CudaShardKernels`` is the
product: it calls the C ABI on this process's GPU), so the exchange can be
exercised on CPU processes with the gloo backend and a stand-in kernel
object.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import HytError, check, lib
from .graph import _ptr


@dataclass
class PageRankVectors:
    """Whole-graph vectors of one sharded PageRank solve."""

    rank: list          # two float32 [V]
    contrib: list       # two float32 [V]
    sums: object        # float64 [2]: L1 change, dangling mass (this shard's rows, then all)
    damping: float
    personalized: bool = False
    source: int = 0     # caller's vertex id (personalized)


class CudaShardKernels:
    """The shard entry points of the C ABI for one process: shard `part` of
    `parts` of `graph`, with its vectors on the graph's GPU."""

    def __init__(self, graph, part: int, parts: int):
        import torch

        self.torch = torch
        self.graph = graph
        self.part, self.parts = int(part), int(parts)
        self.num_vertices = int(graph.num_vertices)
        self.device = torch.device("cuda", getattr(graph, "device", torch.cuda.current_device()))
        self._bounds = {}
        self._shards = {}

    # -- layout --------------------------------------------------------------
    def _bounds_array(self, kind: int) -> np.ndarray:
        if kind not in self._bounds:
            b = np.zeros(self.parts + 1, np.uint32)
            check(lib.hyt_shard_bounds(self.graph.handle, kind, self.parts, _ptr(b)))
            self._bounds[kind] = b
        return self._bounds[kind]

    def bounds(self, kind: int) -> list:
        return [int(x) for x in self._bounds_array(kind)]

    def _shard(self, kind: int) -> C.c_void_p:
        if kind not in self._shards:
            b = self._bounds_array(kind)
            h = C.c_void_p()
            check(lib.hyt_shard_create(self.graph.handle, kind, _ptr(b), self.parts, self.part, C.byref(h)))
            self._shards[kind] = h
        return self._shards[kind]

    def info(self, kind: int) -> dict:
        i = capi.hyt_shard_info()
        check(lib.hyt_shard_get_info(self._shard(kind), C.byref(i)))
        return i.as_dict()

    def empty(self, n: int, dtype):
        return self.torch.empty(n, dtype=dtype, device=self.device)

    def _stream(self) -> int:
        """torch's current stream; its legacy default stream (handle 0) goes
        over as cudaStreamLegacy (1), because NULL selects the graph's own
        stream, which torch's reads of the vectors would not wait for."""
        return self.torch.cuda.current_stream(self.device).cuda_stream or 1

    # -- PageRank ------------------------------------------------------------
    def _pr_args(self, v: PageRankVectors) -> capi.hyt_shard_pagerank:
        a = capi.hyt_shard_pagerank()
        a.rank[0], a.rank[1] = _ptr(v.rank[0]), _ptr(v.rank[1])
        a.contrib[0], a.contrib[1] = _ptr(v.contrib[0]), _ptr(v.contrib[1])
        a.sums = _ptr(v.sums)
        a.damping = v.damping
        a.personalized = 1 if v.personalized else 0
        a.source = int(v.source)
        a.stream = self._stream()
        return a

    def pagerank_init(self, v: PageRankVectors) -> None:
        a = self._pr_args(v)
        check(lib.hyt_shard_pagerank_init(self._shard(capi.HYT_SHARD_PULL), C.byref(a)))

    def pagerank_step(self, v: PageRankVectors, iteration: int, dangling: float) -> None:
        a = self._pr_args(v)
        check(lib.hyt_shard_pagerank_step(self._shard(capi.HYT_SHARD_PULL), C.byref(a), iteration, dangling))

    def emit(self, values, out=None):
        """Internal-order float32 [V] (every entry current) in caller order,
        into out (host or device; a new numpy array by default)."""
        out = np.empty(self.num_vertices, np.float32) if out is None else out
        check(lib.hyt_shard_emit(self._shard(capi.HYT_SHARD_PULL), _ptr(values), _ptr(out), self._stream()))
        return out

    # -- SSSP ----------------------------------------------------------------
    def _ss_args(self, keys, source: int = 0, frontier=None) -> capi.hyt_shard_sssp:
        return capi.hyt_shard_sssp(_ptr(keys), int(source), 0, self._stream(), _ptr(frontier) or None)

    def sssp_init(self, keys, source: int) -> None:
        a = self._ss_args(keys, source)
        check(lib.hyt_shard_sssp_init(self._shard(capi.HYT_SHARD_PUSH), C.byref(a)))

    def sssp_collect(self, keys, frontier) -> None:
        """This shard's frontier of the round; its out-edge count into
        frontier (int64 [1])."""
        a = self._ss_args(keys, frontier=frontier)
        check(lib.hyt_shard_sssp_collect(self._shard(capi.HYT_SHARD_PUSH), C.byref(a)))

    def sssp_relax(self, keys, frontier) -> None:
        """Push (or, when the summed frontier count in `frontier` is dense,
        pull-sweep) relaxations into keys; keys[V] = this shard's idle flag."""
        a = self._ss_args(keys, frontier=frontier)
        check(lib.hyt_shard_sssp_relax(self._shard(capi.HYT_SHARD_PUSH), C.byref(a)))

    def sssp_labels(self, keys, out=None):
        out = np.empty(self.num_vertices, np.uint32) if out is None else out
        check(lib.hyt_shard_sssp_labels(self._shard(capi.HYT_SHARD_PUSH), _ptr(keys), _ptr(out),
                                        self._stream()))
        return out

    def close(self) -> None:
        for h in self._shards.values():
            check(lib.hyt_shard_destroy(h))
        self._shards = {}


class ShardedGraph:
    """A graph solved by all processes of a torch.distributed group, one
    vertex range each.  Every process passes the same graph (same CSR, same
    flags); with no initialised process group it is a single shard.

    ``kernels`` replaces the C-ABI kernels (tests use a CPU stand-in)."""

    def __init__(self, graph=None, group=None, kernels=None):
        import torch.distributed as dist

        self.group = group
        self.dist = dist if (dist.is_available() and dist.is_initialized()) else None
        self.part = self.dist.get_rank(group) if self.dist else 0
        self.parts = self.dist.get_world_size(group) if self.dist else 1
        if kernels is None:
            if graph is None:
                raise ValueError("ShardedGraph needs a graph (or kernels)")
            kernels = CudaShardKernels(graph, self.part, self.parts)
        self.kernels = kernels
        self.num_vertices = int(kernels.num_vertices)

    # -- exchange ------------------------------------------------------------
    def _owner(self, p: int) -> int:
        return self.dist.get_global_rank(self.group, p) if self.group is not None else p

    def _share_slices(self, vec, bounds) -> int:
        """Every process receives every owner's slice of vec: one all-gather
        of slices padded to the longest, then one gather back into place.
        Returns the vector's bytes (4 per vertex for float32), the payload
        every process ends up holding."""
        if self.dist is None:
            return 0
        import torch

        P = self.parts
        sizes = [bounds[p + 1] - bounds[p] for p in range(P)]
        m = max(sizes)
        if m == 0:
            return 0
        key = (tuple(bounds), vec.device, vec.dtype)
        if getattr(self, "_gather_key", None) != key:
            # idx[v] = position of vertex v in the padded all-gather buffer
            owner = np.repeat(np.arange(P), sizes)
            starts = np.asarray(bounds[:-1], np.int64)
            idx = owner * m + (np.arange(bounds[-1], dtype=np.int64) - starts[owner])
            self._gather_idx = torch.from_numpy(idx).to(vec.device)
            self._gather_send = torch.zeros(m, dtype=vec.dtype, device=vec.device)
            self._gather_recv = torch.empty(P * m, dtype=vec.dtype, device=vec.device)
            self._gather_key = key
        lo, hi = bounds[self.part], bounds[self.part + 1]
        self._gather_send[: hi - lo].copy_(vec[lo:hi])
        self.dist.all_gather_into_tensor(self._gather_recv, self._gather_send, group=self.group)
        torch.index_select(self._gather_recv, 0, self._gather_idx, out=vec[: bounds[-1]])
        return sum(sizes) * vec.element_size()

    def _sum(self, t) -> None:
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)

    def _min(self, t) -> None:
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)

    # -- solvers -------------------------------------------------------------
    def _pull(self, damping: float, tolerance: float, max_iterations: int, personalized: bool, source: int, out):
        import torch

        if not (math.isfinite(tolerance) and tolerance > 0):
            raise HytError(capi.HYT_E_INVALID, "PageRank tolerance must be finite and positive")
        if max_iterations <= 0:
            raise HytError(capi.HYT_E_INVALID, "PageRank max_iterations must be greater than zero")
        k = self.kernels
        V = self.num_vertices
        bounds = k.bounds(capi.HYT_SHARD_PULL)
        v = PageRankVectors(rank=[k.empty(V, torch.float32) for _ in range(2)],
                            contrib=[k.empty(V, torch.float32) for _ in range(2)],
                            sums=k.empty(2, torch.float64), damping=float(damping),
                            personalized=personalized, source=int(source))
        tol = float(np.float32(tolerance))  # the stop rule compares with the float tolerance
        t0 = time.perf_counter()
        k.pagerank_init(v)
        self._sum(v.sums)
        dangling = float(v.sums[1].item())
        moved, iterations, residual, converged = 0, 0, 0.0, False
        for it in range(int(max_iterations)):
            k.pagerank_step(v, it, dangling)
            moved += self._share_slices(v.contrib[(it + 1) & 1], bounds)
            self._sum(v.sums)
            residual, dangling = (float(x) for x in v.sums.tolist())
            iterations = it + 1
            if residual <= tol:
                converged = True
                break
        final = v.rank[iterations & 1]
        moved += self._share_slices(final, bounds)
        ranks = k.emit(final, out)
        ms = 1e3 * (time.perf_counter() - t0)
        return ranks, {"iterations": iterations, "converged": int(converged), "residual": residual, "ms": ms,
                       "part": self.part, "parts": self.parts, "vertex_begin": bounds[self.part],
                       "vertex_end": bounds[self.part + 1], "exchanged_bytes": moved}

    def pagerank(self, damping: float = 0.85, tolerance: float = 1e-6, max_iterations: int = 100, out=None):
        """Ranks float32 [V] (caller order, on every process) and stats; out:
        a host or device array to receive them (a new numpy array by
        default)."""
        return self._pull(damping, tolerance, max_iterations, False, 0, out)

    def ppr(self, source: int, restart: float = 0.15, tolerance: float = 1e-6, max_iterations: int = 100,
            out=None):
        if not (0.0 < restart <= 1.0):
            raise HytError(capi.HYT_E_INVALID, "personalized PageRank restart must be in (0, 1]")
        damping = float(np.float32(1.0) - np.float32(restart))  # 1 - restart in float, as hyt_ppr forms it
        return self._pull(damping, tolerance, max_iterations, True, source, out)

    def sssp(self, source: int, max_rounds: int = 0, out=None):
        """Labels uint32 [V] (caller order, on every process) and stats; the
        rounds stop at the fixed point, or at max_rounds when given."""
        import torch

        k = self.kernels
        V = self.num_vertices
        cap = int(max_rounds) if max_rounds else min(4 * V + 1024, 0x7FFFFFFF)
        keys = k.empty(V + 1, torch.int32)
        frontier = k.empty(1, torch.int64)
        t0 = time.perf_counter()
        k.sssp_init(keys, source)
        rounds, converged = 0, False
        while rounds < cap:
            k.sssp_collect(keys, frontier)
            self._sum(frontier)  # one push / pull decision for all shards
            k.sssp_relax(keys, frontier)
            self._min(keys)
            rounds += 1
            if int(keys[V].item()) == 1:
                converged = True
                break
        labels = k.sssp_labels(keys, out)
        ms = 1e3 * (time.perf_counter() - t0)
        bounds = k.bounds(capi.HYT_SHARD_PUSH)
        return labels, {"iterations": rounds, "converged": int(converged), "ms": ms, "part": self.part,
                        "parts": self.parts, "vertex_begin": bounds[self.part], "vertex_end": bounds[self.part + 1],
                        "exchanged_bytes": (4 * (V + 1) + 8) * rounds if self.dist else 0}

    def close(self) -> None:
        close = getattr(self.kernels, "close", None)
        if close:
            close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
