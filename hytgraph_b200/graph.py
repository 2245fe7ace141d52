"""Python host API over the C ABI: CSR containers, the seeded R-MAT
generator, and a device-resident graph handle with PageRank / personalized
PageRank / SSSP solvers.

Arrays may be numpy arrays (host) or any object exposing ``data_ptr()`` and
``numel()`` (e.g. torch CUDA tensors) for device-resident inputs/outputs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import capi
from .capi import HytError, check, lib

RMAT_A, RMAT_B, RMAT_C = 0.57, 0.19, 0.19


def _ptr(x) -> int:
    if x is None:
        return 0
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return int(x.ctypes.data)
    raise TypeError(f"unsupported array type {type(x)!r}")


@dataclass
class CSR:
    """Host CSR: row_offsets uint64[V+1], column_indices uint32[E], weights
    uint32[E] / float32[E] / None."""

    row_offsets: np.ndarray
    column_indices: np.ndarray
    weights: Optional[np.ndarray] = None

    @property
    def num_vertices(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def num_edges(self) -> int:
        return int(self.column_indices.shape[0])

    @property
    def weight_kind(self) -> int:
        if self.weights is None:
            return capi.HYT_WEIGHTS_NONE
        return capi.HYT_WEIGHTS_F32 if self.weights.dtype == np.float32 else capi.HYT_WEIGHTS_U32

    def out_degree(self) -> np.ndarray:
        return np.diff(self.row_offsets)

    def to_c(self) -> capi.hyt_csr:
        if self.row_offsets.dtype != np.uint64 or self.column_indices.dtype != np.uint32:
            raise TypeError("row_offsets must be uint64 and column_indices uint32")
        if self.weights is not None and self.weights.dtype not in (np.uint32, np.float32):
            raise TypeError("weights must be uint32 or float32")
        c = capi.hyt_csr()
        c.num_vertices = self.num_vertices
        c.num_edges = self.num_edges
        c.row_offsets = _ptr(self.row_offsets)
        c.column_indices = _ptr(self.column_indices) if self.num_edges else 0
        c.weights = _ptr(self.weights) if (self.weights is not None and self.num_edges) else 0
        c.weight_kind = self.weight_kind
        return c


@dataclass
class DeviceCSR:
    """A CSR whose arrays live in device memory (owned by the library)."""

    buffers: capi.hyt_csr_buffers
    weight_kind: int = capi.HYT_WEIGHTS_U32  # of the weights, when present

    @property
    def num_vertices(self) -> int:
        return int(self.buffers.num_vertices)

    @property
    def num_edges(self) -> int:
        return int(self.buffers.num_edges)

    def to_c(self) -> capi.hyt_csr:
        b = self.buffers
        c = capi.hyt_csr()
        c.num_vertices = b.num_vertices
        c.num_edges = b.num_edges
        c.row_offsets = C.cast(b.row_offsets, C.c_void_p).value
        c.column_indices = C.cast(b.column_indices, C.c_void_p).value
        c.weights = C.cast(b.weights, C.c_void_p).value if b.weights else 0
        c.weight_kind = self.weight_kind if b.weights else capi.HYT_WEIGHTS_NONE
        return c

    def download(self, row_offsets=None, column_indices=None, weights=None) -> CSR:
        """Copies the device arrays into host arrays (numpy by default, or
        caller-provided buffers such as pinned tensors viewed as numpy)."""
        V, E = self.num_vertices, self.num_edges
        b = self.buffers
        off = np.empty(V + 1, np.uint64) if row_offsets is None else row_offsets
        cols = np.empty(E, np.uint32) if column_indices is None else column_indices
        w = None
        if b.weights:
            w = np.empty(E, np.float32 if self.weight_kind == capi.HYT_WEIGHTS_F32 else np.uint32) \
                if weights is None else weights
        capi.copy(_ptr(off), C.cast(b.row_offsets, C.c_void_p).value, (V + 1) * 8)
        if E:
            capi.copy(_ptr(cols), C.cast(b.column_indices, C.c_void_p).value, E * 4)
            if w is not None:
                capi.copy(_ptr(w), C.cast(b.weights, C.c_void_p).value, E * 4)
        return CSR(off, cols, w)

    def free(self) -> None:
        check(lib.hyt_csr_buffers_free(C.byref(self.buffers)))

    def __del__(self):
        try:
            if self.buffers.row_offsets:
                lib.hyt_csr_buffers_free(C.byref(self.buffers))
        except Exception:
            pass


def rmat_params(scale: int, edge_factor: int, seed: int, weight_min: int = 1, weight_max: int = 63,
                a: float = RMAT_A, b: float = RMAT_B, c: float = RMAT_C) -> capi.hyt_rmat_params:
    p = capi.hyt_rmat_params()
    p.scale, p.edge_factor, p.seed = scale, edge_factor, seed
    p.a, p.b, p.c = a, b, c
    p.weight_min, p.weight_max = weight_min, weight_max
    return p


def rmat(scale: int, edge_factor: int, seed: int, weight_min: int = 1, weight_max: int = 63,
         a: float = RMAT_A, b: float = RMAT_B, c: float = RMAT_C, device: bool = False):
    """Seeded R-MAT graph (self-loops and duplicates removed, sorted by
    (source, destination)).  Host: returns CSR of numpy copies.  device=True:
    generated on the GPU and returned as a DeviceCSR."""
    p = rmat_params(scale, edge_factor, seed, weight_min, weight_max, a, b, c)
    buf = capi.hyt_csr_buffers()
    check(lib.hyt_rmat_generate(C.byref(p), 1 if device else 0, C.byref(buf)))
    if device:
        return DeviceCSR(buf)
    try:
        V, E = int(buf.num_vertices), int(buf.num_edges)
        off = np.ctypeslib.as_array(buf.row_offsets, shape=(V + 1,)).copy()
        cols = np.ctypeslib.as_array(buf.column_indices, shape=(max(E, 1),))[:E].copy()
        w = None
        if buf.weights:
            w = np.ctypeslib.as_array(buf.weights, shape=(max(E, 1),))[:E].copy()
    finally:
        check(lib.hyt_csr_buffers_free(C.byref(buf)))
    return CSR(off, cols, w)


def pick_sources(row_offsets: np.ndarray, seed: int, count: int) -> np.ndarray:
    """`count` seeded vertices with out-degree > 0 (distinct while possible)."""
    ro = np.ascontiguousarray(row_offsets, dtype=np.uint64)
    out = np.zeros(count, dtype=np.uint32)
    check(lib.hyt_pick_sources(_ptr(ro), ro.shape[0] - 1, seed, count, _ptr(out)))
    return out


class Graph:
    """Device-resident graph (hyt_graph handle)."""

    def __init__(self, csr, flags: int = capi.HYT_GRAPH_ALL, device: Optional[int] = None, stream: int = 0):
        """device: CUDA ordinal; None = the calling thread's current device
        (the one torch.cuda.set_device chose, as one process per GPU needs)."""
        self._csr_ref = csr  # keep host arrays alive during creation
        opts = capi.hyt_graph_options(flags, -1 if device is None else device, stream or None)
        c = csr.to_c()
        h = C.c_void_p()
        check(lib.hyt_graph_create(C.byref(c), C.byref(opts), C.byref(h)))
        self._h = h
        self.device = int(self.info()["device"])
        self.num_vertices = int(c.num_vertices)
        self.num_edges = int(c.num_edges)
        self._csr_ref = None

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("graph is closed")
        return self._h

    def info(self) -> dict:
        i = capi.hyt_graph_info()
        check(lib.hyt_graph_get_info(self.handle, C.byref(i)))
        return {name: getattr(i, name) for name, _ in i._fields_}

    def pagerank(self, damping: float = 0.85, tolerance: float = 1e-6, max_iterations: int = 100,
                 out=None, flags: int = 0, stream: int = 0):
        p = capi.hyt_pagerank_params(damping, tolerance, max_iterations, flags, stream or None)
        st = capi.hyt_run_stats()
        res = np.empty(self.num_vertices, dtype=np.float32) if out is None else out
        check(lib.hyt_pagerank(self.handle, C.byref(p), _ptr(res) if res is not False else None, C.byref(st)))
        return res, st.as_dict()

    def ppr(self, source: int, restart: float = 0.15, tolerance: float = 1e-6, max_iterations: int = 100,
            out=None, flags: int = 0, stream: int = 0):
        p = capi.hyt_ppr_params(source, restart, tolerance, max_iterations, flags, stream or None)
        st = capi.hyt_run_stats()
        res = np.empty(self.num_vertices, dtype=np.float32) if out is None else out
        check(lib.hyt_ppr(self.handle, C.byref(p), _ptr(res) if res is not False else None, C.byref(st)))
        return res, st.as_dict()

    def ppr_multi(self, sources, restart: float = 0.15, tolerance: float = 1e-6, max_iterations: int = 100,
                  out=None):
        """Personalized PageRank of 1-8 sources in one packed solve
        (hyt_ppr_multi): returns (ranks float32 [k][V], per-query stats)."""
        src = np.ascontiguousarray(sources, np.uint32)
        k = int(src.shape[0])
        res = np.empty((k, self.num_vertices), dtype=np.float32) if out is None else out
        st = (capi.hyt_run_stats * max(k, 1))()
        check(lib.hyt_ppr_multi(self.handle, _ptr(src) if k else None, k, restart, tolerance, max_iterations,
                                _ptr(res) if res is not False else None, st))
        return res, [st[i].as_dict() for i in range(k)]

    def sssp_multi(self, sources, max_rounds: int = 0, out=None):
        """SSSP of 1-8 sources in one shared solve (hyt_sssp_multi): returns
        (labels uint32 [k][V], stats of the call)."""
        src = np.ascontiguousarray(sources, np.uint32)
        k = int(src.shape[0])
        res = np.empty((k, self.num_vertices), dtype=np.uint32) if out is None else out
        st = capi.hyt_run_stats()
        check(lib.hyt_sssp_multi(self.handle, _ptr(src) if k else None, k, max_rounds,
                                 _ptr(res) if res is not False else None, C.byref(st)))
        return res, st.as_dict()

    def pagerank_contributions(self, current_ranks, damping: float = 0.85, out=None):
        """|next - current| of one synchronous PageRank pull step per vertex
        (hyt_pagerank_contributions); float64 [V], numpy or a CUDA tensor."""
        cur = np.ascontiguousarray(current_ranks, np.float32) if isinstance(current_ranks, np.ndarray) else current_ranks
        res = np.empty(self.num_vertices, np.float64) if out is None else out
        check(lib.hyt_pagerank_contributions(self.handle, _ptr(cur), damping, _ptr(res)))
        return res

    def sssp(self, source: int, out=None, flags: int = 0, max_rounds: int = 0, delta: int = 0, stream: int = 0):
        p = capi.hyt_sssp_params(source, delta, max_rounds, flags, stream or None)
        st = capi.hyt_run_stats()
        res = np.empty(self.num_vertices, dtype=np.uint32) if out is None else out
        check(lib.hyt_sssp(self.handle, C.byref(p), _ptr(res) if res is not False else None, C.byref(st)))
        return res, st.as_dict()

    def copy_csc(self, in_offsets=None, in_sources=None):
        """The graph's CSC (ascending sources per in-row) into host numpy
        arrays, or caller buffers (host or device)."""
        off = np.empty(self.num_vertices + 1, np.uint64) if in_offsets is None else in_offsets
        src = np.empty(max(self.num_edges, 1), np.uint32) if in_sources is None else in_sources
        check(lib.hyt_graph_copy_csc(self.handle, _ptr(off), _ptr(src)))
        return off, (src[: self.num_edges] if in_sources is None else src)

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib.hyt_graph_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedBuffer:
    """Pinned, device-mapped host memory (hyt_pinned_alloc) viewed as numpy."""

    def __init__(self, count: int, dtype):
        self.dtype = np.dtype(dtype)
        self.count = int(count)
        p = C.c_void_p()
        check(lib.hyt_pinned_alloc(max(self.count, 1) * self.dtype.itemsize, C.byref(p)))
        self._p = p.value
        buf = (C.c_char * (max(self.count, 1) * self.dtype.itemsize)).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=self.count)

    def data_ptr(self) -> int:
        return self._p

    def free(self) -> None:
        if getattr(self, "_p", None):
            self.array = None
            check(lib.hyt_pinned_free(self._p))
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def pinned_copy(x: np.ndarray) -> PinnedBuffer:
    b = PinnedBuffer(x.shape[0], x.dtype)
    if x.shape[0]:
        b.array[:] = x
    return b


class HybridGraph:
    """Graph whose edges stay in pinned host memory (hyt_hybrid handle):
    the CSR (push, SSSP) and CSC (pull, PageRank) edge arrays are read per
    partition through resident HBM copies, staged copies, host compaction
    or zero-copy, as the HyTM cost model decides.

    Arrays are numpy (copied into pinned buffers that this object owns) or
    PinnedBuffer objects (used in place); they must outlive the handle."""

    def __init__(self, row_offsets, column_indices, weights=None, in_offsets=None, in_sources=None,
                 flags: int = capi.HYT_GRAPH_ALL, device: Optional[int] = None, budget_bytes: int = 0,
                 partition_vertices: int = 0, host_threads: int = 0, force_engine: int = capi.HYT_ENGINE_AUTO,
                 alpha: float = 0.0, beta: float = 0.0, gamma: float = 0.0):
        def pin(x):
            if x is None or isinstance(x, PinnedBuffer):
                return x
            return pinned_copy(np.ascontiguousarray(x))

        self._bufs = [pin(x) for x in (row_offsets, column_indices, weights, in_offsets, in_sources)]
        off, cols, w, ioff, isrc = self._bufs
        V = off.count - 1
        E = cols.count
        c = capi.hyt_csr(V, E, off.data_ptr(), cols.data_ptr(), w.data_ptr() if w is not None else None,
                         capi.HYT_WEIGHTS_U32 if w is not None else capi.HYT_WEIGHTS_NONE)
        cc = None
        if ioff is not None:
            cc = capi.hyt_csc(V, isrc.count, ioff.data_ptr(), isrc.data_ptr())
        opts = capi.hyt_hybrid_options(flags, -1 if device is None else device, budget_bytes, partition_vertices,
                                       host_threads, force_engine,
                                       alpha, beta, gamma)
        h = C.c_void_p()
        check(lib.hyt_hybrid_create(C.byref(c), C.byref(cc) if cc is not None else None, C.byref(opts),
                                    C.byref(h)))
        self._h = h
        self.num_vertices = V
        self.num_edges = E

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("hybrid graph is closed")
        return self._h

    def info(self) -> dict:
        i = capi.hyt_hybrid_info()
        check(lib.hyt_hybrid_get_info(self.handle, C.byref(i)))
        return i.as_dict()

    def pagerank(self, damping: float = 0.85, tolerance: float = 1e-6, max_iterations: int = 100, out=None):
        p = capi.hyt_pagerank_params(damping, tolerance, max_iterations, 0, None)
        st, ts = capi.hyt_run_stats(), capi.hyt_hybrid_stats()
        res = np.empty(self.num_vertices, dtype=np.float32) if out is None else out
        check(lib.hyt_hybrid_pagerank(self.handle, C.byref(p), _ptr(res) if res is not False else None,
                                      C.byref(st), C.byref(ts)))
        return res, st.as_dict(), ts.as_dict()

    def sssp(self, source: int, out=None, max_rounds: int = 0):
        p = capi.hyt_sssp_params(source, 0, max_rounds, 0, None)
        st, ts = capi.hyt_run_stats(), capi.hyt_hybrid_stats()
        res = np.empty(self.num_vertices, dtype=np.uint32) if out is None else out
        check(lib.hyt_hybrid_sssp(self.handle, C.byref(p), _ptr(res) if res is not False else None,
                                  C.byref(st), C.byref(ts)))
        return res, st.as_dict(), ts.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib.hyt_hybrid_destroy(self._h))
            self._h = None
        self._bufs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many SSSP / personalized-PageRank queries over many resident graphs,
    run together (hyt_batch handle): one CUDA-graph launch per batch.

    queries: sequence of (graph_index, kind, source) or dicts with keys
    graph, kind ("sssp" | "ppr" or HYT_QUERY_*), source, and optionally
    restart, tolerance, max_iterations, out (an array to receive the result;
    by default a numpy array is allocated per query)."""

    def __init__(self, graphs, device: Optional[int] = None, state_budget_bytes: int = 0, delta_mult: int = 0,
                 hub_degree: int = 0, ctas_per_sm: int = 0, flags: int = 0):
        self._graphs = list(graphs)  # keep the graph handles alive
        if device is None:  # the graphs' device
            device = self._graphs[0].device if self._graphs else -1
        arr = (C.c_void_p * len(self._graphs))(*[g.handle.value for g in self._graphs])
        opts = capi.hyt_batch_options(device, state_budget_bytes,
                                      capi.hyt_batch_tuning(delta_mult, hub_degree, ctas_per_sm), flags)
        h = C.c_void_p()
        check(lib.hyt_batch_create(arr, len(self._graphs), C.byref(opts), C.byref(h)))
        self._h = h

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("batch is closed")
        return self._h

    def _pack(self, queries, with_out: bool = True):
        n = len(queries)
        arr = (capi.hyt_query * n)()
        outs = []
        for i, q in enumerate(queries):
            if not isinstance(q, dict):
                q = {"graph": q[0], "kind": q[1], "source": q[2]}
            kind = q["kind"]
            if isinstance(kind, str):
                kind = capi.HYT_QUERY_SSSP if kind == "sssp" else capi.HYT_QUERY_PPR
            gi = q["graph"]
            g = self._graphs[gi] if 0 <= gi < len(self._graphs) else None  # the library rejects bad indices
            out = q.get("out")
            if out is None and with_out and g is not None:
                out = np.empty(g.num_vertices, np.uint32 if kind == capi.HYT_QUERY_SSSP else np.float32)
            outs.append(out)
            arr[i] = capi.hyt_query(q["graph"], kind, q["source"], q.get("restart", 0.0), q.get("tolerance", 0.0),
                                    q.get("max_iterations", 0), _ptr(out) if out is not None else None)
        return arr, outs

    def run(self, queries):
        """Returns (outputs, per-query result dicts, batch stats dict)."""
        arr, outs = self._pack(queries)
        n = len(queries)
        res = (capi.hyt_query_result * max(n, 1))()
        st = capi.hyt_batch_stats()
        check(lib.hyt_batch_run(self.handle, arr, n, res, C.byref(st)))
        return outs, [res[i].as_dict() for i in range(n)], st.as_dict()

    def autotune(self, queries) -> dict:
        arr, _ = self._pack(queries, with_out=False)
        t = capi.hyt_batch_tuning()
        check(lib.hyt_batch_autotune(self.handle, arr, len(queries), C.byref(t)))
        return t.as_dict()

    def set_tuning(self, delta_mult: int = 0, hub_degree: int = 0, ctas_per_sm: int = 0) -> None:
        t = capi.hyt_batch_tuning(delta_mult, hub_degree, ctas_per_sm)
        check(lib.hyt_batch_set_tuning(self.handle, C.byref(t)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib.hyt_batch_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching query server (hyt_server handle): submit() from
    any thread, poll() for completions.  A query's `out` array must stay
    alive until its completion has been polled."""

    def __init__(self, graphs, device: Optional[int] = None, state_budget_bytes: int = 0, delta_mult: int = 0,
                 hub_degree: int = 0, ctas_per_sm: int = 0, max_running: int = 0, pack_min_edges: int = 0):
        self._graphs = list(graphs)
        if device is None:  # the graphs' device
            device = self._graphs[0].device if self._graphs else -1
        arr = (C.c_void_p * len(self._graphs))(*[g.handle.value for g in self._graphs])
        opts = capi.hyt_server_options(device, state_budget_bytes,
                                       capi.hyt_batch_tuning(delta_mult, hub_degree, ctas_per_sm), max_running,
                                       pack_min_edges)
        h = C.c_void_p()
        check(lib.hyt_server_create(arr, len(self._graphs), C.byref(opts), C.byref(h)))
        self._h = h
        self._outs = {}

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("server is closed")
        return self._h

    def submit(self, graph: int, kind, source: int, out=None, restart: float = 0.0, tolerance: float = 0.0,
               max_iterations: int = 0) -> int:
        if isinstance(kind, str):
            kind = capi.HYT_QUERY_SSSP if kind == "sssp" else capi.HYT_QUERY_PPR
        if out is None and 0 <= graph < len(self._graphs):
            out = np.empty(self._graphs[graph].num_vertices, np.uint32 if kind == capi.HYT_QUERY_SSSP else np.float32)
        q = capi.hyt_query(graph, kind, source, restart, tolerance, max_iterations,
                           _ptr(out) if out is not None else None)
        t = C.c_uint64()
        check(lib.hyt_server_submit(self.handle, C.byref(q), C.byref(t)))
        self._outs[t.value] = out
        return t.value

    def poll(self, max_items: int = 1024, wait_ms: int = 0):
        """List of completion dicts: ticket, status, result, queue_ms,
        latency_ms, out (the array holding the result)."""
        buf = (capi.hyt_completion * max_items)()
        n = C.c_uint32()
        check(lib.hyt_server_poll(self.handle, buf, max_items, C.byref(n), wait_ms))
        out = []
        for i in range(n.value):
            c = buf[i]
            out.append({"ticket": c.ticket, "status": c.status, "result": c.result.as_dict(),
                        "queue_ms": c.queue_ms, "latency_ms": c.latency_ms, "out": self._outs.pop(c.ticket, None)})
        return out

    def stats(self) -> dict:
        st = capi.hyt_server_stats()
        check(lib.hyt_server_get_stats(self.handle, C.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib.hyt_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hub_sort(csr, hub_fraction: float = 0.08, order_out=None, scores_out=None, stats: Optional[dict] = None):
    """Hub-first vertex order on the GPU (hyt_hub_sort): returns
    (vertex_order uint32[V], scores float64[V], hub_count).  csr: CSR or
    DeviceCSR.  order_out / scores_out: optional caller buffers (numpy, or
    CUDA tensors to keep the results on the device; scores_out=False skips
    the scores).  stats: filled with the call's device figures."""
    c = csr.to_c()
    V = int(c.num_vertices)
    order = np.empty(V, np.uint32) if order_out is None else order_out
    scores = np.empty(V, np.float64) if scores_out is None else scores_out
    n = C.c_uint64()
    st = capi.hyt_reorder_stats()
    check(lib.hyt_hub_sort(C.byref(c), hub_fraction, _ptr(order) if V else None,
                           _ptr(scores) if (scores is not False and V) else None, C.byref(n), C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return order, scores, n.value


def reorder(csr, vertex_order, device: bool = False, stats: Optional[dict] = None):
    """CSRGraph::reorder_vertices on the GPU (hyt_csr_reorder): a host CSR,
    or a DeviceCSR when device=True.  vertex_order: numpy or a CUDA tensor."""
    c = csr.to_c()
    if isinstance(vertex_order, (np.ndarray, list, tuple)):
        order = np.ascontiguousarray(vertex_order, np.uint32)
        shape = order.shape
    else:
        order = vertex_order
        shape = tuple(order.shape)
    if shape != (csr.num_vertices,):
        raise HytError(capi.HYT_E_INVALID,
                       "CSRGraph::reorder_vertices: vertex_order must contain exactly one entry per vertex")
    b = capi.hyt_csr_buffers()
    st = capi.hyt_reorder_stats()
    check(lib.hyt_csr_reorder(C.byref(c), _ptr(order) if csr.num_vertices else None, 1 if device else 0,
                              C.byref(b), C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    if device:
        return DeviceCSR(b, csr.weight_kind)
    return _host_csr(b)


def _host_csr(b) -> "CSR":
    """Host CSR of numpy copies of library-allocated host buffers (freed)."""
    V, E = int(b.num_vertices), int(b.num_edges)
    off = np.ctypeslib.as_array(b.row_offsets, shape=(V + 1,)).copy()
    cols = np.ctypeslib.as_array(b.column_indices, shape=(max(E, 1),))[:E].copy() if E else np.zeros(0, np.uint32)
    w = None
    if b.weights:
        wa = np.ctypeslib.as_array(b.weights, shape=(max(E, 1),))[:E].copy() if E else np.zeros(0, np.uint32)
        w = wa.view(np.float32) if b.weight_kind == capi.HYT_WEIGHTS_F32 else wa
    check(lib.hyt_csr_buffers_free(C.byref(b)))
    return CSR(off, cols, w)


def _wrap(b, device: bool):
    return DeviceCSR(b, int(b.weight_kind) or capi.HYT_WEIGHTS_U32) if device else _host_csr(b)


def load_edge_list(path, num_vertices: int, weighted: bool = False, device: bool = False,
                   stats: Optional[dict] = None):
    """GraphLoader::load_edge_list (hyt_load_edge_list): a text edge list ->
    CSR (float weights when weighted), or a DeviceCSR when device=True."""
    b, st = capi.hyt_csr_buffers(), capi.hyt_load_stats()
    check(lib.hyt_load_edge_list(str(path).encode(), num_vertices, 1 if weighted else 0, 1 if device else 0,
                                 C.byref(b), C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return _wrap(b, device)


def csr_from_edges(src, dst, num_vertices: int, weights=None, device: bool = False, stats: Optional[dict] = None):
    """CSR of an edge array on the GPU (hyt_csr_from_edges): edges grouped by
    source in input order, parallel edges kept.  Arrays: numpy or CUDA
    tensors; weights uint32 / float32 (or int32 / float32 tensors)."""
    def arr(x, dt):
        return np.ascontiguousarray(x, dt) if isinstance(x, (np.ndarray, list, tuple)) else x
    s, d = arr(src, np.uint32), arr(dst, np.uint32)
    E = int(s.shape[0])
    if tuple(d.shape) != (E,) or (weights is not None and tuple(weights.shape) != (E,)):
        raise HytError(capi.HYT_E_INVALID, "src, dst and weights must have one entry per edge")
    kind = capi.HYT_WEIGHTS_NONE
    if weights is not None:
        is_f32 = str(getattr(weights, "dtype", "")).endswith("float32")
        kind = capi.HYT_WEIGHTS_F32 if is_f32 else capi.HYT_WEIGHTS_U32
        if isinstance(weights, np.ndarray) and not is_f32:
            weights = np.ascontiguousarray(weights, np.uint32)
    b, st = capi.hyt_csr_buffers(), capi.hyt_load_stats()
    check(lib.hyt_csr_from_edges(_ptr(s) if E else None, _ptr(d) if E else None,
                                 _ptr(weights) if (weights is not None and E) else None, kind, E, num_vertices,
                                 1 if device else 0, C.byref(b), C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return _wrap(b, device)


def save_csr(csr, path) -> None:
    """Writes the binary CSR file (hyt_csr_save); csr: CSR or DeviceCSR."""
    c = csr.to_c()
    check(lib.hyt_csr_save(str(path).encode(), C.byref(c)))


def load_csr(path, device: bool = False, stats: Optional[dict] = None):
    """Reads a binary CSR file (hyt_csr_load), checking its checksum and
    structure: a CSR, or a DeviceCSR when device=True."""
    b, st = capi.hyt_csr_buffers(), capi.hyt_load_stats()
    check(lib.hyt_csr_load(str(path).encode(), 1 if device else 0, C.byref(b), C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return _wrap(b, device)


def sssp_contributions(current, candidate, tolerance: float = 0.0, out=None):
    """sssp_contributions on the GPU (hyt_sssp_contributions): float64 [n]."""
    c = np.ascontiguousarray(current, np.float32) if isinstance(current, np.ndarray) else current
    d = np.ascontiguousarray(candidate, np.float32) if isinstance(candidate, np.ndarray) else candidate
    n = int(c.shape[0])
    if tuple(d.shape) != (n,):
        raise HytError(capi.HYT_E_INVALID, "SSSP contribution distance vectors must have equal size")
    res = np.empty(n, np.float64) if out is None else out
    check(lib.hyt_sssp_contributions(_ptr(c) if n else None, _ptr(d) if n else None, n, tolerance,
                                     _ptr(res) if n else None))
    return res


def contribution_schedule(items, contributions, deterministic_tie_break: bool = True,
                          zero_contribution_epsilon: float = 0.0, out=None):
    """ContributionScheduler::schedule on the GPU (hyt_contribution_schedule):
    returns (ordered item indices uint64 [n], metrics dict)."""
    it = np.ascontiguousarray(items, np.uint64) if not hasattr(items, "data_ptr") else items
    c = np.ascontiguousarray(contributions, np.float64) if not hasattr(contributions, "data_ptr") else contributions
    n = int(it.shape[0])
    if tuple(c.shape) != (n,):
        raise HytError(capi.HYT_E_INVALID, "contribution priority inputs must have equal size")
    res = np.empty(n, np.uint64) if out is None else out
    m = capi.hyt_contribution_metrics()
    check(lib.hyt_contribution_schedule(_ptr(it) if n else None, _ptr(c) if n else None, n,
                                        1 if deterministic_tie_break else 0, zero_contribution_epsilon,
                                        _ptr(res) if n else None, C.byref(m)))
    return res, m.as_dict()


def partition_contributions(vertex_contributions, bounds, out=None):
    """Per-partition sums of vertex contributions over [bounds[i], bounds[i+1])
    (hyt_partition_contributions): the priorities of the transfer queue."""
    c = np.ascontiguousarray(vertex_contributions, np.float64) if isinstance(vertex_contributions, np.ndarray) \
        else vertex_contributions
    b = np.ascontiguousarray(bounds, np.uint64) if not hasattr(bounds, "data_ptr") else bounds
    parts = int(b.shape[0]) - 1
    res = np.empty(max(parts, 0), np.float64) if out is None else out
    check(lib.hyt_partition_contributions(_ptr(c), int(c.shape[0]), _ptr(b), max(parts, 0),
                                          _ptr(res) if parts > 0 else None))
    return res
