#pragma once
// ImpTM-Zero-Copy: kernels read active rows straight from mapped pinned host
// memory.  Source-compatible with hytgraph::transfer::ImpTMZeroCopy
// (reference include/transfer/zero_copy_engine.hpp:15-144).  prepare()
// returns the same request/alignment metrics as the reference's model; the
// executing engine (transfer/hybrid_engine.hpp) performs the real mapped
// reads and reports mode = MappedHost.

#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::transfer {

enum class ZeroCopyMode { Modeled, MappedHost };

struct ZeroCopyVertexMetrics {
    graph::CSRGraph::vertex_id vertex = 0;
    graph::CSRGraph::offset_type degree = 0;
    std::uint64_t memory_requests = 0;     // ceil(degree * 4 / payload)
    std::uint64_t alignment_overhead = 0;  // 1 if the row start is unaligned
};

struct ZeroCopyPartition {
    std::size_t partition_index = 0;
    graph::CSRGraph::vertex_id vertex_begin = 0;
    graph::CSRGraph::vertex_id vertex_end = 0;
    std::vector<graph::CSRGraph::vertex_id> active_vertices;
    std::vector<ZeroCopyVertexMetrics> vertex_metrics;
    graph::CSRGraph::offset_type active_edge_count = 0;
    std::uint64_t memory_request_count = 0;
    std::uint64_t alignment_overhead_count = 0;
    std::uint64_t modeled_tlp_count = 0;
};

struct ZeroCopyResult {
    ZeroCopyMode mode = ZeroCopyMode::Modeled;
    std::vector<ZeroCopyPartition> partitions;
    std::size_t active_partition_count = 0;
    graph::CSRGraph::offset_type active_vertex_count = 0;
    graph::CSRGraph::offset_type active_edge_count = 0;
    std::uint64_t memory_request_count = 0;
    std::uint64_t alignment_overhead_count = 0;
    std::uint64_t modeled_tlp_count = 0;
    bool host_memory_mapped = false;
    double preparation_seconds = 0.0;
};

struct ZeroCopyOptions {
    std::size_t request_payload_bytes = 128U;
    std::size_t max_requests_per_tlp = 256U;
    bool enable_host_mapping = true;
    std::size_t alignment_bytes = 128U;
};

class ImpTMZeroCopy {
public:
    explicit ImpTMZeroCopy(ZeroCopyOptions options = {}) noexcept : options_(options) {}
    [[nodiscard]] const ZeroCopyOptions &options() const noexcept { return options_; }
    // Metrics over the logical byte layout of the CSR (row_offsets[v] * 4);
    // throws std::invalid_argument / std::out_of_range on bad input.
    [[nodiscard]] ZeroCopyResult prepare(const graph::CSRGraph &graph,
                                         const std::vector<graph::LogicalPartition> &partitions,
                                         const graph::ActivityTracker &activity) const;

private:
    ZeroCopyOptions options_;
};

}  // namespace hytgraph::transfer
