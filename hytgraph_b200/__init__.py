"""hytgraph_b200 -- B200-native hybrid-transfer graph processing.

PageRank (pull over CSC), personalized PageRank and frontier SSSP as
hand-written sm_100a CUDA behind a C ABI (include/hyt/capi.h), with the
reference's C++ interfaces (include/graph, include/algorithms,
include/transfer, include/scheduling, include/runtime) in libhytgraph.so.

ShardedGraph runs PageRank / personalized PageRank / SSSP over all GPUs of
a torch.distributed group, one vertex range per process.

Importing the package loads lib/libhyt_core.so and fails if it is missing;
there is no CPU fallback.
"""
from . import capi
from .capi import HytError, device_count, measure_peaks
from .graph import (CSR, Batch, DeviceCSR, Graph, HybridGraph, PinnedBuffer, Server, contribution_schedule,
                    csr_from_edges, hub_sort, load_csr, load_edge_list, partition_contributions, pick_sources, reorder,
                    rmat, save_csr, sssp_contributions)
from .shard import CudaShardKernels, ShardedGraph

__all__ = [
    "capi", "HytError", "device_count", "measure_peaks", "CSR", "Batch", "DeviceCSR", "Graph", "HybridGraph", "PinnedBuffer", "Server",
    "contribution_schedule", "csr_from_edges", "hub_sort", "load_csr", "load_edge_list", "partition_contributions",
    "pick_sources", "reorder", "rmat", "save_csr", "sssp_contributions", "CudaShardKernels", "ShardedGraph",
]
