"""ctypes bindings of the C ABI in include/hyt/capi.h (libhyt_core.so).

The library is loaded from hytgraph_b200/lib/ (built in-tree by
``make -C hytgraph_b200``).  There is no fallback: if the shared library is
missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
CORE_PATH = LIB_DIR / "libhyt_core.so"

HYT_OK = 0
HYT_E_INVALID = 1
HYT_E_CUDA = 2
HYT_E_OOM = 3
HYT_E_TIMEOUT = 4
HYT_E_NO_DEVICE = 5
HYT_E_UNSUPPORTED = 6
HYT_E_INTERNAL = 7
HYT_E_IO = 8

HYT_WEIGHTS_NONE = 0
HYT_WEIGHTS_U32 = 1
HYT_WEIGHTS_F32 = 2

HYT_GRAPH_PULL = 1
HYT_GRAPH_PUSH = 2
HYT_GRAPH_ALL = 3
HYT_GRAPH_HUB_ORDER = 4

HYT_RUN_PROFILE = 1
HYT_RUN_NO_GRAPH = 2

HYT_DIST_INF_U32 = 0xFFFFFFFF
HYT_SHARD_PULL = 1  # vertex-range shard kinds (hyt_shard_bounds / hyt_shard_create)
HYT_SHARD_PUSH = 2
HYT_NOALLOC_MAX_VERTICES = 1 << 20  # hyt_sssp_noalloc capacity (include/hyt/capi.h)
HYT_NOALLOC_MAX_EDGES = 1 << 24


class hyt_csr(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("row_offsets", C.c_void_p),
        ("column_indices", C.c_void_p),
        ("weights", C.c_void_p),
        ("weight_kind", C.c_uint32),
    ]


class hyt_graph_options(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("device", C.c_int), ("stream", C.c_void_p)]


class hyt_graph_info(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("weight_kind", C.c_uint32),
        ("flags", C.c_uint32),
        ("device_bytes", C.c_uint64),
        ("pull_tiles", C.c_uint64),
        ("long_rows", C.c_uint64),
        ("max_in_degree", C.c_uint64),
        ("max_out_degree", C.c_uint64),
        ("dangling_vertices", C.c_uint64),
        ("build_ms", C.c_double),
        ("device", C.c_int32),
        ("pad", C.c_uint32),
    ]


class hyt_pagerank_params(C.Structure):
    _fields_ = [
        ("damping", C.c_float),
        ("tolerance", C.c_float),
        ("max_iterations", C.c_uint32),
        ("flags", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class hyt_ppr_params(C.Structure):
    _fields_ = [
        ("source", C.c_uint32),
        ("restart", C.c_float),
        ("tolerance", C.c_float),
        ("max_iterations", C.c_uint32),
        ("flags", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class hyt_run_stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("converged", C.c_uint32),
        ("residual", C.c_double),
        ("device_ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("kernel_launches", C.c_uint32),
        ("total_launches", C.c_uint32),
        ("edges_processed", C.c_uint64),
        ("vertices_processed", C.c_uint64),
        ("algorithmic_bytes", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_sssp_params(C.Structure):
    _fields_ = [
        ("source", C.c_uint32),
        ("delta", C.c_uint32),
        ("max_rounds", C.c_uint32),
        ("flags", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class hyt_rmat_params(C.Structure):
    _fields_ = [
        ("scale", C.c_uint32),
        ("edge_factor", C.c_uint32),
        ("a", C.c_double),
        ("b", C.c_double),
        ("c", C.c_double),
        ("seed", C.c_uint64),
        ("weight_min", C.c_uint32),
        ("weight_max", C.c_uint32),
    ]


class hyt_csr_buffers(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("row_offsets", C.POINTER(C.c_uint64)),
        ("column_indices", C.POINTER(C.c_uint32)),
        ("weights", C.POINTER(C.c_uint32)),
        ("on_device", C.c_uint32),
        ("weight_kind", C.c_uint32),
    ]


class hyt_reorder_stats(C.Structure):
    _fields_ = [
        ("device_ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("kernel_bytes", C.c_uint64),
        ("algorithmic_bytes", C.c_uint64),
        ("kernel_launches", C.c_uint32),
        ("library_calls", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_load_stats(C.Structure):
    _fields_ = [
        ("total_ms", C.c_double),
        ("read_ms", C.c_double),
        ("device_ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("file_bytes", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("kernel_bytes", C.c_uint64),
        ("threads", C.c_uint32),
        ("pad", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


class hyt_contribution_metrics(C.Structure):
    _fields_ = [
        ("input_item_count", C.c_uint64),
        ("scheduled_item_count", C.c_uint64),
        ("reordered_item_count", C.c_uint64),
        ("zero_contribution_count", C.c_uint64),
        ("scheduling_overhead", C.c_double),
        ("stale_work_count", C.c_uint64),
        ("redundant_work_count", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_csc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64),
        ("num_edges", C.c_uint64),
        ("in_offsets", C.c_void_p),
        ("in_sources", C.c_void_p),
    ]


HYT_ENGINE_AUTO = 0
HYT_ENGINE_FILTER = 1
HYT_ENGINE_COMPACTION = 2
HYT_ENGINE_ZERO_COPY = 3


class hyt_hybrid_options(C.Structure):
    _fields_ = [
        ("flags", C.c_uint32),
        ("device", C.c_int),
        ("device_budget_bytes", C.c_uint64),
        ("partition_vertices", C.c_uint32),
        ("host_threads", C.c_uint32),
        ("force_engine", C.c_uint32),
        ("alpha", C.c_float),
        ("beta", C.c_float),
        ("gamma", C.c_float),
    ]


class hyt_hybrid_info(C.Structure):
    _fields_ = [
        ("partitions", C.c_uint64),
        ("budget_bytes", C.c_uint64),
        ("resident_bytes", C.c_uint64),
        ("staging_bytes", C.c_uint64),
        ("resident_push_partitions", C.c_uint64),
        ("resident_pull_partitions", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("h2d_gbs", C.c_double),
        ("zero_copy_gbs", C.c_double),
        ("gather_gbs", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_hybrid_stats(C.Structure):
    _fields_ = [
        ("rounds", C.c_uint64),
        ("resident_decisions", C.c_uint64),
        ("filter_decisions", C.c_uint64),
        ("compaction_decisions", C.c_uint64),
        ("zero_copy_decisions", C.c_uint64),
        ("filter_bytes", C.c_uint64),
        ("compaction_bytes", C.c_uint64),
        ("zero_copy_bytes", C.c_uint64),
        ("link_bytes", C.c_uint64),
        ("necessary_bytes", C.c_uint64),
        ("copies", C.c_uint64),
        ("compaction_host_ms", C.c_double),
        ("device_ms", C.c_double),
        ("link_gbs", C.c_double),
        ("h2d_peak_gbs", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


HYT_QUERY_SSSP = 0
HYT_QUERY_PPR = 1


class hyt_query(C.Structure):
    _fields_ = [
        ("graph", C.c_uint32),
        ("kind", C.c_uint32),
        ("source", C.c_uint32),
        ("restart", C.c_float),
        ("tolerance", C.c_float),
        ("max_iterations", C.c_uint32),
        ("out", C.c_void_p),
    ]


class hyt_query_result(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("converged", C.c_uint32),
        ("residual", C.c_double),
        ("edges_processed", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_batch_tuning(C.Structure):
    _fields_ = [
        ("delta_mult", C.c_uint32),
        ("hub_degree", C.c_uint32),
        ("ctas_per_sm", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_batch_options(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("state_budget_bytes", C.c_uint64),
        ("tuning", hyt_batch_tuning),
        ("flags", C.c_uint32),
    ]


class hyt_batch_stats(C.Structure):
    _fields_ = [
        ("device_ms", C.c_double),
        ("supersteps", C.c_uint32),
        ("waves", C.c_uint32),
        ("graph_launches", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("edges_processed", C.c_uint64),
        ("algorithmic_bytes", C.c_uint64),
        ("state_bytes", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_server_options(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("state_budget_bytes", C.c_uint64),
        ("tuning", hyt_batch_tuning),
        ("max_running", C.c_uint32),
        ("pack_min_edges", C.c_uint32),
    ]


class hyt_completion(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("status", C.c_int),
        ("result", hyt_query_result),
        ("queue_ms", C.c_double),
        ("latency_ms", C.c_double),
    ]


class hyt_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("supersteps", C.c_uint64),
        ("graph_launches", C.c_uint64),
        ("running", C.c_uint32),
        ("waiting", C.c_uint32),
        ("max_running", C.c_uint32),
        ("state_bytes", C.c_uint64),
        ("peak_state_bytes", C.c_uint64),
        ("busy_ms", C.c_double),
        ("packs", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class hyt_shard_info(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("part", C.c_uint32),
        ("parts", C.c_uint32),
        ("vertex_begin", C.c_uint32),
        ("vertex_end", C.c_uint32),
        ("pad", C.c_uint32),
        ("num_vertices", C.c_uint64),
        ("edges", C.c_uint64),
        ("tasks", C.c_uint64),
        ("edges_relaxed", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


class hyt_shard_pagerank(C.Structure):
    _fields_ = [
        ("rank", C.c_void_p * 2),
        ("contrib", C.c_void_p * 2),
        ("sums", C.c_void_p),
        ("damping", C.c_float),
        ("personalized", C.c_uint32),
        ("source", C.c_uint32),
        ("pad", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class hyt_shard_sssp(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("source", C.c_uint32), ("pad", C.c_uint32), ("stream", C.c_void_p),
                ("frontier_edges", C.c_void_p)]


class hyt_peaks(C.Structure):
    _fields_ = [
        ("hbm_copy_gbs", C.c_double),
        ("h2d_gbs", C.c_double),
        ("d2h_gbs", C.c_double),
        ("zero_copy_gbs", C.c_double),
        ("hbm_bytes", C.c_uint64),
        ("l2_bytes", C.c_uint64),
        ("copy_bytes", C.c_uint64),
        ("link_bytes", C.c_uint64),
        ("sm_count", C.c_uint32),
        ("mem_bus_bits", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class HytError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[hyt status {code}] {message}")
        self.code = code


# (name, restype, argtypes)
_SIGNATURES = [
    ("hyt_last_error", C.c_char_p, []),
    ("hyt_abi_version", C.c_int, []),
    ("hyt_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("hyt_copy", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("hyt_graph_create", C.c_int, [C.POINTER(hyt_csr), C.POINTER(hyt_graph_options), C.POINTER(C.c_void_p)]),
    ("hyt_graph_destroy", C.c_int, [C.c_void_p]),
    ("hyt_graph_get_info", C.c_int, [C.c_void_p, C.POINTER(hyt_graph_info)]),
    ("hyt_pagerank", C.c_int, [C.c_void_p, C.POINTER(hyt_pagerank_params), C.c_void_p, C.POINTER(hyt_run_stats)]),
    ("hyt_ppr", C.c_int, [C.c_void_p, C.POINTER(hyt_ppr_params), C.c_void_p, C.POINTER(hyt_run_stats)]),
    ("hyt_sssp", C.c_int, [C.c_void_p, C.POINTER(hyt_sssp_params), C.c_void_p, C.POINTER(hyt_run_stats)]),
    ("hyt_sssp_noalloc", C.c_int, [C.POINTER(hyt_csr), C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(hyt_run_stats)]),
    ("hyt_graph_copy_csc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hyt_pinned_alloc", C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
    ("hyt_pinned_free", C.c_int, [C.c_void_p]),
    ("hyt_hybrid_create", C.c_int,
     [C.POINTER(hyt_csr), C.POINTER(hyt_csc), C.POINTER(hyt_hybrid_options), C.POINTER(C.c_void_p)]),
    ("hyt_hybrid_destroy", C.c_int, [C.c_void_p]),
    ("hyt_hybrid_get_info", C.c_int, [C.c_void_p, C.POINTER(hyt_hybrid_info)]),
    ("hyt_hybrid_pagerank", C.c_int,
     [C.c_void_p, C.POINTER(hyt_pagerank_params), C.c_void_p, C.POINTER(hyt_run_stats), C.POINTER(hyt_hybrid_stats)]),
    ("hyt_hybrid_sssp", C.c_int,
     [C.c_void_p, C.POINTER(hyt_sssp_params), C.c_void_p, C.POINTER(hyt_run_stats), C.POINTER(hyt_hybrid_stats)]),
    ("hyt_batch_create", C.c_int,
     [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(hyt_batch_options), C.POINTER(C.c_void_p)]),
    ("hyt_batch_destroy", C.c_int, [C.c_void_p]),
    ("hyt_batch_run", C.c_int,
     [C.c_void_p, C.POINTER(hyt_query), C.c_uint32, C.POINTER(hyt_query_result), C.POINTER(hyt_batch_stats)]),
    ("hyt_batch_autotune", C.c_int, [C.c_void_p, C.POINTER(hyt_query), C.c_uint32, C.POINTER(hyt_batch_tuning)]),
    ("hyt_batch_set_tuning", C.c_int, [C.c_void_p, C.POINTER(hyt_batch_tuning)]),
    ("hyt_server_create", C.c_int,
     [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(hyt_server_options), C.POINTER(C.c_void_p)]),
    ("hyt_server_submit", C.c_int, [C.c_void_p, C.POINTER(hyt_query), C.POINTER(C.c_uint64)]),
    ("hyt_server_poll", C.c_int,
     [C.c_void_p, C.POINTER(hyt_completion), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
    ("hyt_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(hyt_server_stats)]),
    ("hyt_server_destroy", C.c_int, [C.c_void_p]),
    ("hyt_hub_sort", C.c_int, [C.POINTER(hyt_csr), C.c_double, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64),
                               C.POINTER(hyt_reorder_stats)]),
    ("hyt_load_edge_list", C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.c_int, C.POINTER(hyt_csr_buffers),
                                     C.POINTER(hyt_load_stats)]),
    ("hyt_csr_from_edges", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_int,
                                     C.POINTER(hyt_csr_buffers), C.POINTER(hyt_load_stats)]),
    ("hyt_csr_save", C.c_int, [C.c_char_p, C.POINTER(hyt_csr)]),
    ("hyt_csr_load", C.c_int, [C.c_char_p, C.c_int, C.POINTER(hyt_csr_buffers), C.POINTER(hyt_load_stats)]),
    ("hyt_pagerank_contributions", C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]),
    ("hyt_sssp_contributions", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_float, C.c_void_p]),
    ("hyt_contribution_schedule", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_double, C.c_void_p,
                                            C.POINTER(hyt_contribution_metrics)]),
    ("hyt_partition_contributions", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("hyt_trim_device_memory", C.c_int, [C.c_int]),
    ("hyt_sssp_multi", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                 C.POINTER(hyt_run_stats)]),
    ("hyt_ppr_multi", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.c_void_p,
                                C.POINTER(hyt_run_stats)]),
    ("hyt_csr_reorder", C.c_int, [C.POINTER(hyt_csr), C.c_void_p, C.c_int, C.POINTER(hyt_csr_buffers),
                                  C.POINTER(hyt_reorder_stats)]),
    ("hyt_rmat_generate", C.c_int, [C.POINTER(hyt_rmat_params), C.c_int, C.POINTER(hyt_csr_buffers)]),
    ("hyt_csr_buffers_free", C.c_int, [C.POINTER(hyt_csr_buffers)]),
    ("hyt_pick_sources", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p]),
    ("hyt_measure_peaks", C.c_int, [C.c_int, C.c_uint64, C.POINTER(hyt_peaks)]),
    ("hyt_shard_bounds", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]),
    ("hyt_shard_create", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                   C.POINTER(C.c_void_p)]),
    ("hyt_shard_destroy", C.c_int, [C.c_void_p]),
    ("hyt_shard_get_info", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_info)]),
    ("hyt_shard_pagerank_init", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_pagerank)]),
    ("hyt_shard_pagerank_step", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_pagerank), C.c_uint32, C.c_double]),
    ("hyt_shard_sssp_init", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_sssp)]),
    ("hyt_shard_sssp_collect", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_sssp)]),
    ("hyt_shard_sssp_relax", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_sssp)]),
    ("hyt_shard_sssp_round", C.c_int, [C.c_void_p, C.POINTER(hyt_shard_sssp)]),
    ("hyt_shard_sssp_labels", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hyt_shard_emit", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
]

EXPORTED = [name for name, _, _ in _SIGNATURES]


def _load() -> C.CDLL:
    if not CORE_PATH.exists():
        raise ImportError(
            f"{CORE_PATH} is missing: build it with `make -C {CORE_PATH.parent.parent}` "
            "(or __graft_entry__.build()); there is no CPU fallback"
        )
    lib = C.CDLL(str(CORE_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
    for name, res, args in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.hyt_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status != HYT_OK:
        raise HytError(status, last_error())


def copy(dst: int, src: int, nbytes: int, stream: int = 0) -> None:
    """Synchronous copy between host/device addresses (integers)."""
    check(lib.hyt_copy(dst, src, nbytes, stream or None))


def measure_peaks(device: int = 0, copy_bytes: int = 0) -> dict:
    """Measured HBM copy, pinned host-link and zero-copy bandwidths of one
    GPU (hyt_measure_peaks), GB/s, plus its memory and SM facts."""
    p = hyt_peaks()
    check(lib.hyt_measure_peaks(device, copy_bytes, C.byref(p)))
    return p.as_dict()


def device_count() -> int:
    n = C.c_int(0)
    check(lib.hyt_device_count(C.byref(n)))
    return n.value
