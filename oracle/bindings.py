"""ctypes access to the oracle (liboracle.so, the C restatement) and to the
reference's own compiled CPU code (_ref/libhytref.so, optional).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU legs of bench.py, as the checker / CPU baseline.  The product
package never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libhytref.so"

u64p = C.POINTER(C.c_uint64)


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref when the reference sources exist)."""
    subprocess.run(["make", "-C", str(HERE)], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class HytmOptions(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double), ("rtt", C.c_double),
                ("cpu_throughput", C.c_double), ("m", C.c_uint64), ("mr", C.c_uint64), ("d1", C.c_uint64),
                ("d2", C.c_uint64), ("align", C.c_uint64)]


class HytmCosts(C.Structure):
    _fields_ = [("active_vertices", C.c_uint64), ("active_edges", C.c_uint64), ("total_edges", C.c_uint64),
                ("filter_bytes", C.c_uint64), ("compaction_bytes", C.c_uint64), ("zc_requests", C.c_uint64),
                ("zc_alignment", C.c_uint64), ("filter_cost", C.c_double), ("compaction_cost", C.c_double),
                ("zero_copy_cost", C.c_double), ("zc_rtt", C.c_double), ("engine", C.c_int)]


class Oracle:
    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        self.lib = C.CDLL(str(ORACLE_SO))

    def pagerank_f32(self, off, cols, damping=0.85, tol=1e-6, max_iter=100):
        V, E = off.shape[0] - 1, cols.shape[0]
        r = np.empty(V, np.float32)
        it, res, conv = C.c_uint64(), C.c_float(), C.c_int()
        rc = self.lib.oracle_pagerank_f32(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_float(damping),
                                          C.c_float(tol), C.c_uint64(max_iter), _p(r), C.byref(it), C.byref(res),
                                          C.byref(conv))
        if rc:
            raise ValueError(f"oracle_pagerank_f32 rc={rc}")
        return r, it.value, res.value, bool(conv.value)

    def pagerank_f64(self, off, cols, damping=0.85, tol=1e-6, max_iter=100):
        V, E = off.shape[0] - 1, cols.shape[0]
        r = np.empty(V, np.float64)
        it, res, conv = C.c_uint64(), C.c_double(), C.c_int()
        rc = self.lib.oracle_pagerank_f64(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_double(damping),
                                          C.c_double(tol), C.c_uint64(max_iter), _p(r), C.byref(it), C.byref(res),
                                          C.byref(conv))
        if rc:
            raise ValueError(f"oracle_pagerank_f64 rc={rc}")
        return r, it.value, res.value, bool(conv.value)

    def pagerank_f64_csc(self, off, in_off, in_src, damping=0.85, tol=1e-6, max_iter=100):
        """pagerank_f64 on a given incoming CSR (sources ascending per row)."""
        V = off.shape[0] - 1
        r = np.empty(V, np.float64)
        it, res, conv = C.c_uint64(), C.c_double(), C.c_int()
        rc = self.lib.oracle_pagerank_f64_csc(C.c_uint64(V), _p(off), _p(in_off), _p(in_src), C.c_double(damping),
                                              C.c_double(tol), C.c_uint64(max_iter), _p(r), C.byref(it),
                                              C.byref(res), C.byref(conv))
        if rc:
            raise ValueError(f"oracle_pagerank_f64_csc rc={rc}")
        return r, it.value, res.value, bool(conv.value)

    def ppr_f64(self, off, cols, source, restart=0.15, tol=1e-6, max_iter=100):
        V, E = off.shape[0] - 1, cols.shape[0]
        r = np.empty(V, np.float64)
        it, res, conv = C.c_uint64(), C.c_double(), C.c_int()
        rc = self.lib.oracle_ppr_f64(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_uint32(source),
                                     C.c_double(restart), C.c_double(tol), C.c_uint64(max_iter), _p(r),
                                     C.byref(it), C.byref(res), C.byref(conv))
        if rc:
            raise ValueError(f"oracle_ppr_f64 rc={rc}")
        return r, it.value, res.value, bool(conv.value)

    def sssp(self, off, cols, weights_f32, source, max_iter=0):
        V, E = off.shape[0] - 1, cols.shape[0]
        d = np.empty(V, np.float32)
        it, conv = C.c_uint64(), C.c_int()
        rc = self.lib.oracle_sssp(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), _p(weights_f32),
                                  C.c_uint32(source), C.c_uint64(max_iter), _p(d), C.byref(it), C.byref(conv))
        if rc:
            raise ValueError(f"oracle_sssp rc={rc}")
        return d, it.value, bool(conv.value)

    def dijkstra(self, off, cols, weights_u32, source):
        V, E = off.shape[0] - 1, cols.shape[0]
        d = np.empty(V, np.uint64)
        rc = self.lib.oracle_dijkstra_u32(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), _p(weights_u32),
                                          C.c_uint32(source), _p(d))
        if rc:
            raise ValueError(f"oracle_dijkstra_u32 rc={rc}")
        return d

    def rmat(self, scale, edge_factor, seed, weight_min=1, weight_max=63, a=0.57, b=0.19, c=0.19):
        """Seeded R-MAT CSR (the same bytes as the product's generator):
        (row_offsets uint64[V+1], column_indices uint32[E], weights uint32[E]
        or None)."""
        off_p, cols_p, w_p = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        E = C.c_uint64()
        rc = self.lib.oracle_rmat(C.c_uint32(scale), C.c_uint32(edge_factor), C.c_uint64(seed), C.c_double(a),
                                  C.c_double(b), C.c_double(c), C.c_uint32(weight_min), C.c_uint32(weight_max),
                                  C.byref(off_p), C.byref(cols_p), C.byref(w_p), C.byref(E))
        if rc:
            raise ValueError(f"oracle_rmat rc={rc}")
        V, E = 1 << scale, E.value
        try:
            off = np.ctypeslib.as_array(off_p, shape=(V + 1,)).copy()
            cols = np.ctypeslib.as_array(cols_p, shape=(max(E, 1),))[:E].copy()
            w = np.ctypeslib.as_array(w_p, shape=(max(E, 1),))[:E].copy() if w_p else None
        finally:
            for p in (off_p, cols_p, w_p):
                if p:
                    self.lib.oracle_free(p)
        return off, cols, w

    def pick_sources(self, off, seed, count):
        out = np.zeros(max(count, 1), np.uint32)
        rc = self.lib.oracle_pick_sources(_p(np.ascontiguousarray(off, np.uint64)), C.c_uint64(off.shape[0] - 1),
                                          C.c_uint64(seed), C.c_uint32(count), _p(out))
        if rc:
            raise ValueError(f"oracle_pick_sources rc={rc}")
        return out[:count]

    def hytm_partition(self, off, active_u8, vbegin, vend, opts: HytmOptions) -> HytmCosts:
        c = HytmCosts()
        self.lib.oracle_hytm_partition(_p(off), _p(active_u8), C.c_uint32(vbegin), C.c_uint32(vend),
                                       C.byref(opts), C.byref(c))
        return c

    def select_engine(self, f, c, z, alpha, beta) -> int:
        self.lib.oracle_select_engine.restype = C.c_int
        return self.lib.oracle_select_engine(C.c_double(f), C.c_double(c), C.c_double(z), C.c_double(alpha),
                                             C.c_double(beta))

    def task_combine(self, engines, k):
        e = np.ascontiguousarray(engines, dtype=np.int32)
        n = e.shape[0]
        top = np.zeros(max(n, 1), np.uint64)
        teng = np.zeros(max(n, 1) + 2, np.int32)
        tfirst = np.zeros(max(n, 1) + 2, np.uint64)
        self.lib.oracle_task_combine.restype = C.c_uint64
        nt = self.lib.oracle_task_combine(_p(e), C.c_uint64(n), C.c_uint64(k), _p(top), _p(teng), _p(tfirst))
        return top[:n], teng[:nt], tfirst[:nt]


    def hub_sort(self, off, cols, fraction=0.08):
        V, E = off.shape[0] - 1, cols.shape[0]
        order = np.empty(max(V, 1), np.uint32)
        scores = np.empty(max(V, 1), np.float64)
        n = C.c_uint64()
        rc = self.lib.oracle_hub_sort(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_double(fraction),
                                      _p(order), _p(scores), C.byref(n))
        if rc:
            raise ValueError(f"oracle_hub_sort rc={rc}")
        return order[:V], scores[:V], n.value

    def reorder(self, off, cols, w, order):
        """w: any 4-byte weight array or None; returns (offsets, columns, weights)."""
        V, E = off.shape[0] - 1, cols.shape[0]
        o = np.empty(V + 1, np.uint64)
        c = np.empty(max(E, 1), np.uint32)
        wo = np.empty(max(E, 1), np.uint32) if w is not None else None
        rc = self.lib.oracle_reorder(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols),
                                     _p(w.view(np.uint32)) if w is not None else None,
                                     _p(np.ascontiguousarray(order, np.uint32)), _p(o), _p(c), _p(wo))
        if rc:
            raise ValueError(f"oracle_reorder rc={rc}")
        return o, c[:E], (wo[:E].view(w.dtype) if w is not None else None)

    LOAD_ERRORS = {1: "unable to open file: {path}", 2: "malformed edge at line {line}",
                   3: "vertex ID out of range at line {line}", 4: "missing edge weight at line {line}",
                   5: "unexpected data at line {line}"}

    def load_edge_list(self, path, V, weighted):
        """GraphLoader::load_edge_list restated; returns (offsets, columns,
        weights or None) or raises ValueError with the reference's message."""
        E, line = C.c_uint64(), C.c_uint64()
        rc = self.lib.oracle_load_edge_list(str(path).encode(), C.c_uint64(V), C.c_int(1 if weighted else 0),
                                            C.byref(E), C.byref(line))
        if rc:
            raise ValueError("GraphLoader::load_edge_list: " + self.LOAD_ERRORS[rc].format(path=path, line=line.value))
        o = np.empty(V + 1, np.uint64)
        c = np.empty(max(E.value, 1), np.uint32)
        w = np.empty(max(E.value, 1), np.float32) if weighted else None
        self.lib.oracle_loaded_copy(_p(o), _p(c), _p(w) if w is not None else None)
        self.lib.oracle_loaded_free()
        return o, c[:E.value], (w[:E.value] if w is not None else None)

    def csr_from_edges(self, V, src, dst, w=None):
        E = int(src.shape[0])
        o = np.empty(V + 1, np.uint64)
        c = np.empty(max(E, 1), np.uint32)
        wo = np.empty(max(E, 1), np.uint32) if w is not None else None
        self.lib.oracle_csr_from_edges.restype = C.c_uint64
        bad = self.lib.oracle_csr_from_edges(C.c_uint64(V), C.c_uint64(E), _p(np.ascontiguousarray(src, np.uint32)),
                                             _p(np.ascontiguousarray(dst, np.uint32)),
                                             _p(w.view(np.uint32)) if w is not None else None, _p(o), _p(c), _p(wo))
        if bad:
            raise ValueError(f"edge {bad - 1} has a vertex id >= {V}")
        return o, c[:E], (wo[:E].view(w.dtype) if w is not None else None)

    def pagerank_contributions(self, off, cols, cur, damping=0.85, fp64=False):
        V, E = off.shape[0] - 1, cols.shape[0]
        out = np.empty(V, np.float64)
        rc = self.lib.oracle_pagerank_contributions(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols),
                                                    _p(np.ascontiguousarray(cur, np.float32)), C.c_float(damping),
                                                    C.c_int(1 if fp64 else 0), _p(out))
        if rc:
            raise ValueError(f"oracle_pagerank_contributions rc={rc}")
        return out

    def sssp_contributions(self, cur, cand, tol=0.0):
        n = cur.shape[0]
        out = np.empty(n, np.float64)
        self.lib.oracle_sssp_contributions(C.c_uint64(n), _p(np.ascontiguousarray(cur, np.float32)),
                                           _p(np.ascontiguousarray(cand, np.float32)), C.c_float(tol), _p(out))
        return out

    def contribution_schedule(self, items, contrib, deterministic=True, eps=0.0):
        n = len(items)
        it = np.ascontiguousarray(items, np.uint64)
        c = np.ascontiguousarray(contrib, np.float64)
        out = np.empty(max(n, 1), np.uint64)
        m = np.zeros(7, np.uint64)
        rc = self.lib.oracle_contribution_schedule(C.c_uint64(n), _p(it), _p(c), C.c_int(1 if deterministic else 0),
                                                   C.c_double(eps), _p(out), _p(m))
        if rc:
            raise ValueError("contribution priority must be finite")
        return out[:n], _metrics(m)


def _metrics(m):
    return {"input_item_count": int(m[0]), "scheduled_item_count": int(m[1]), "reordered_item_count": int(m[2]),
            "zero_contribution_count": int(m[3]), "scheduling_overhead": float(m[4:5].view(np.float64)[0]),
            "stale_work_count": int(m[5]), "redundant_work_count": int(m[6])}


class Reference:
    """The reference's own CPU implementation (oracle/_ref/libhytref.so)."""

    def __init__(self):
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources)")
        self.lib = C.CDLL(str(REF_SO))
        self.lib.ref_last_error.restype = C.c_char_p

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def _check(self, rc, what):
        if rc:
            raise ValueError(f"{what} rc={rc}: {self.lib.ref_last_error().decode()}")

    def pagerank_cpu(self, off, cols, damping=0.85, tol=1e-6, max_iter=100):
        V, E = off.shape[0] - 1, cols.shape[0]
        r = np.empty(V, np.float32)
        it, res, conv = C.c_uint64(), C.c_float(), C.c_int()
        self._check(self.lib.ref_pagerank_cpu(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_float(damping),
                                              C.c_float(tol), C.c_uint64(max_iter), _p(r), C.byref(it),
                                              C.byref(res), C.byref(conv)), "ref_pagerank_cpu")
        return r, it.value, res.value, bool(conv.value)

    def sssp_cpu(self, off, cols, weights_f32, source, max_iter=0):
        V, E = off.shape[0] - 1, cols.shape[0]
        d = np.empty(V, np.float32)
        it, conv = C.c_uint64(), C.c_int()
        self._check(self.lib.ref_sssp_cpu(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), _p(weights_f32),
                                          C.c_uint32(source), C.c_uint64(max_iter), _p(d), C.byref(it),
                                          C.byref(conv)), "ref_sssp_cpu")
        return d, it.value, bool(conv.value)

    def hytm_evaluate(self, off, cols, active_u8, parts, dopts, uopts):
        V, E = off.shape[0] - 1, cols.shape[0]
        parts = np.ascontiguousarray(parts, np.uint32)
        n = parts.shape[0]
        metrics = np.zeros((n, 11), np.uint64)
        costs = np.zeros((n, 4), np.float64)
        eng = np.zeros(n, np.int32)
        self._check(self.lib.ref_hytm_evaluate(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), _p(active_u8),
                                               C.c_uint64(n), _p(parts), _p(np.asarray(dopts, np.float64)),
                                               _p(np.asarray(uopts, np.uint64)), _p(metrics), _p(costs), _p(eng)),
                    "ref_hytm_evaluate")
        return metrics, costs, eng

    def select_engine(self, f, c, z, alpha, beta) -> int:
        e = C.c_int()
        self._check(self.lib.ref_select_engine(C.c_double(f), C.c_double(c), C.c_double(z), C.c_double(alpha),
                                               C.c_double(beta), C.byref(e)), "ref_select_engine")
        return e.value

    def task_combine(self, engines, k):
        e = np.ascontiguousarray(engines, dtype=np.int32)
        n = e.shape[0]
        top = np.zeros(max(n, 1), np.uint64)
        teng = np.zeros(max(n, 1) + 2, np.int32)
        tfirst = np.zeros(max(n, 1) + 2, np.uint64)
        nt = C.c_uint64()
        metrics = np.zeros(5, np.uint64)
        self._check(self.lib.ref_task_combine(_p(e), C.c_uint64(n), C.c_uint64(k), _p(top), _p(teng), _p(tfirst),
                                              C.byref(nt), _p(metrics)), "ref_task_combine")
        return top[:n], teng[:nt.value], tfirst[:nt.value], metrics

    def hub_sort(self, off, cols, fraction=0.08):
        V, E = off.shape[0] - 1, cols.shape[0]
        order = np.empty(V, np.uint32)
        scores = np.empty(V, np.float64)
        n = C.c_uint64()
        self._check(self.lib.ref_hub_sort(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols), C.c_double(fraction),
                                          _p(order), _p(scores), C.byref(n)), "ref_hub_sort")
        return order, scores, n.value

    def reorder(self, off, cols, w_f32, order):
        V, E = off.shape[0] - 1, cols.shape[0]
        o = np.empty(V + 1, np.uint64)
        c = np.empty(max(E, 1), np.uint32)
        w = np.empty(max(E, 1), np.float32) if w_f32 is not None else None
        self._check(self.lib.ref_reorder(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols),
                                         _p(w_f32) if w_f32 is not None else None,
                                         _p(np.ascontiguousarray(order, np.uint32)), _p(o), _p(c),
                                         _p(w) if w is not None else None), "ref_reorder")
        return o, c[:E], (w[:E] if w is not None else None)

    def load_edge_list(self, path, V, weighted):
        """GraphLoader::load_edge_list; returns (offsets, columns, weights or None)."""
        E = C.c_uint64()
        self._check(self.lib.ref_load_edge_list(str(path).encode(), C.c_uint64(V), C.c_int(1 if weighted else 0),
                                                C.byref(E)), "ref_load_edge_list")
        o = np.empty(V + 1, np.uint64)
        c = np.empty(max(E.value, 1), np.uint32)
        w = np.empty(max(E.value, 1), np.float32) if weighted else None
        self.lib.ref_loaded_copy(_p(o), _p(c), _p(w) if w is not None else None)
        return o, c[:E.value], (w[:E.value] if w is not None else None)

    def pagerank_contributions(self, off, cols, cur, damping=0.85):
        V, E = off.shape[0] - 1, cols.shape[0]
        out = np.empty(V, np.float64)
        self._check(self.lib.ref_pagerank_contributions(C.c_uint64(V), C.c_uint64(E), _p(off), _p(cols),
                                                        _p(np.ascontiguousarray(cur, np.float32)), C.c_float(damping),
                                                        _p(out)), "ref_pagerank_contributions")
        return out

    def sssp_contributions(self, cur, cand, tol=0.0):
        n = cur.shape[0]
        out = np.empty(n, np.float64)
        self._check(self.lib.ref_sssp_contributions(C.c_uint64(n), _p(np.ascontiguousarray(cur, np.float32)),
                                                    _p(np.ascontiguousarray(cand, np.float32)), C.c_float(tol),
                                                    _p(out)), "ref_sssp_contributions")
        return out

    def contribution_schedule(self, items, contrib, deterministic=True, eps=0.0):
        n = len(items)
        it = np.ascontiguousarray(items, np.uint64)
        c = np.ascontiguousarray(contrib, np.float64)
        out = np.empty(max(n, 1), np.uint64)
        m = np.zeros(7, np.uint64)
        self._check(self.lib.ref_contribution_schedule(C.c_uint64(n), _p(it), _p(c),
                                                       C.c_int(1 if deterministic else 0), C.c_double(eps), _p(out),
                                                       _p(m)), "ref_contribution_schedule")
        return out[:n], _metrics(m)
