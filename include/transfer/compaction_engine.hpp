#pragma once
// ExpTM-Compaction: gather the out-edges of active vertices into a packed
// payload.  Source-compatible with hytgraph::transfer::ExpTMCompaction
// (reference include/transfer/compaction_engine.hpp:26-127).  compact()
// produces the reference's payload layout (active_vertices, neighbors,
// neighbor_index with a leading 0) in O(V + A_e) instead of O(P * V), using
// the host's cores; the executing engine gathers weights too and ships the
// payload with cudaMemcpyAsync on copy streams.

#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"

#include <cstddef>
#include <vector>

namespace hytgraph::transfer {

struct CompactedPartition {
    std::size_t partition_index = 0;
    graph::CSRGraph::vertex_id vertex_begin = 0;
    graph::CSRGraph::vertex_id vertex_end = 0;
    std::vector<graph::CSRGraph::vertex_id> active_vertices;     // ascending
    std::vector<graph::CSRGraph::vertex_id> neighbors;           // packed rows
    std::vector<graph::CSRGraph::offset_type> neighbor_index;    // size A_v + 1

    [[nodiscard]] graph::CSRGraph::offset_type active_edge_count() const noexcept;
    [[nodiscard]] std::size_t active_vertex_count() const noexcept { return active_vertices.size(); }
    [[nodiscard]] std::size_t neighbor_bytes() const noexcept {
        return neighbors.size() * sizeof(graph::CSRGraph::vertex_id);
    }
    [[nodiscard]] std::size_t index_bytes() const noexcept {
        return neighbor_index.size() * sizeof(graph::CSRGraph::offset_type);
    }
    [[nodiscard]] std::size_t total_bytes() const noexcept { return neighbor_bytes() + index_bytes(); }
};

struct CompactionResult {
    std::vector<CompactedPartition> partitions;  // only partitions with an active vertex
    double compaction_seconds = 0.0;             // host wall time of compact()

    [[nodiscard]] std::size_t compacted_partition_count() const noexcept { return partitions.size(); }
    [[nodiscard]] graph::CSRGraph::offset_type active_edge_count() const noexcept;
    [[nodiscard]] graph::CSRGraph::offset_type active_vertex_count() const noexcept;
    [[nodiscard]] std::size_t neighbor_bytes() const noexcept;
    [[nodiscard]] std::size_t index_bytes() const noexcept;
    [[nodiscard]] std::size_t total_bytes() const noexcept;
};

class ExpTMCompaction {
public:
    explicit ExpTMCompaction(bool enabled = true) noexcept : enabled_(enabled) {}
    [[nodiscard]] bool enabled() const noexcept { return enabled_; }
    // Disabled: empty result.  Throws std::invalid_argument for mismatched
    // activity or a partition that is not a CSR row range.
    [[nodiscard]] CompactionResult compact(const graph::CSRGraph &graph,
                                           const std::vector<graph::LogicalPartition> &partitions,
                                           const graph::ActivityTracker &activity) const;
    // The packed destination stream of a compacted partition (validated).
    [[nodiscard]] static std::vector<graph::CSRGraph::vertex_id> expanded_neighbors(
        const CompactedPartition &partition);

private:
    bool enabled_;
};

}  // namespace hytgraph::transfer
