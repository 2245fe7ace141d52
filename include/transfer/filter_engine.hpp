#pragma once
// ExpTM-Filter: whole-partition explicit transfer of every partition that
// holds an active edge.  Source-compatible with hytgraph::transfer::
// ExpTMFilter (reference include/transfer/filter_engine.hpp:13-66).  plan()
// returns the same decisions; the executing engine (transfer/
// hybrid_engine.hpp) turns a "transferred" decision into a cudaMemcpyAsync
// of the partition, or into nothing when the partition is already resident.

#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"

#include <cstddef>
#include <vector>

namespace hytgraph::transfer {

struct FilterPartitionDecision {
    std::size_t partition_index = 0;
    bool active = false;
    bool transferred = false;
    graph::CSRGraph::offset_type active_edges = 0;
    graph::CSRGraph::offset_type total_edges = 0;
    graph::CSRGraph::offset_type transferred_edges = 0;
    std::size_t transferred_bytes = 0;
};

struct FilterTransferPlan {
    std::vector<FilterPartitionDecision> partitions;
    [[nodiscard]] std::size_t active_partition_count() const noexcept;
    [[nodiscard]] std::size_t transferred_partition_count() const noexcept;
    [[nodiscard]] graph::CSRGraph::offset_type transferred_edge_count() const noexcept;
    [[nodiscard]] std::size_t transferred_byte_count() const noexcept;
};

class ExpTMFilter {
public:
    explicit ExpTMFilter(bool enabled = true) noexcept : enabled_(enabled) {}
    [[nodiscard]] bool enabled() const noexcept { return enabled_; }
    // Disabled: every partition is transferred.  Throws std::invalid_argument
    // / std::out_of_range for activity or partitions that do not match.
    [[nodiscard]] FilterTransferPlan plan(const graph::CSRGraph &graph,
                                          const std::vector<graph::LogicalPartition> &partitions,
                                          const graph::ActivityTracker &activity) const;

private:
    bool enabled_;
};

}  // namespace hytgraph::transfer
