#pragma once
// Row-preserving contiguous vertex-range partitions of a CSR graph.
// Source-compatible with hytgraph::graph::LogicalPartition /
// LogicalPartitioner (reference include/graph/partition.hpp:12-84).

#include "graph/csr_graph.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::graph {

class LogicalPartition {
public:
    using vertex_id = CSRGraph::vertex_id;
    using offset_type = CSRGraph::offset_type;
    using byte_type = std::size_t;

    LogicalPartition() = default;
    // Throws std::invalid_argument for begin > end or target_bytes == 0.
    LogicalPartition(vertex_id vertex_begin, vertex_id vertex_end, offset_type edge_begin, offset_type edge_end,
                     byte_type target_bytes);

    [[nodiscard]] vertex_id vertex_begin() const noexcept { return vertex_begin_; }
    [[nodiscard]] vertex_id vertex_end() const noexcept { return vertex_end_; }
    [[nodiscard]] offset_type edge_begin() const noexcept { return edge_begin_; }
    [[nodiscard]] offset_type edge_end() const noexcept { return edge_end_; }
    [[nodiscard]] offset_type vertex_count() const noexcept {
        return static_cast<offset_type>(vertex_end_) - static_cast<offset_type>(vertex_begin_);
    }
    [[nodiscard]] offset_type edge_count() const noexcept { return edge_end_ - edge_begin_; }
    [[nodiscard]] byte_type target_bytes() const noexcept { return target_bytes_; }
    // Bytes of the partition's destination ids only (4 per edge).
    [[nodiscard]] byte_type edge_data_bytes() const noexcept {
        return static_cast<byte_type>(edge_count()) * sizeof(CSRGraph::vertex_id);
    }

private:
    vertex_id vertex_begin_ = 0;
    vertex_id vertex_end_ = 0;
    offset_type edge_begin_ = 0;
    offset_type edge_end_ = 0;
    byte_type target_bytes_ = 0;
};

class LogicalPartitioner {
public:
    using vertex_id = CSRGraph::vertex_id;
    using offset_type = CSRGraph::offset_type;
    using byte_type = std::size_t;

    // 32 MiB of destination ids per partition (HyTGraph's default).
    static constexpr byte_type kDefaultPartitionBytes = 32ULL * 1024ULL * 1024ULL;

    explicit LogicalPartitioner(byte_type partition_bytes = kDefaultPartitionBytes);
    [[nodiscard]] byte_type partition_bytes() const noexcept { return partition_bytes_; }

    // Greedy cut: a partition closes before the first vertex whose row would
    // push its destination-id bytes over the target; a single row larger
    // than the target forms its own (oversized) partition.
    [[nodiscard]] std::vector<LogicalPartition> partition(const CSRGraph &graph) const;

    // Fixed vertex-count partitions (e.g. 2^20 vertices each), the unit of
    // the out-of-HBM transfer engine.  Rows are never split.
    [[nodiscard]] static std::vector<LogicalPartition> partition_by_vertices(const CSRGraph &graph,
                                                                            vertex_id vertices_per_partition);

private:
    byte_type partition_bytes_;
    void check_graph(const CSRGraph &graph) const;
};

}  // namespace hytgraph::graph
