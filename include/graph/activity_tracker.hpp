#pragma once
// Frontier set with HyTGraph's active-subgraph definition: an edge is active
// iff its source vertex is active.  Source-compatible with
// hytgraph::graph::ActivityTracker (reference
// include/graph/activity_tracker.hpp:13-93).

#include "graph/csr_graph.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::graph {

class ActivityTracker {
public:
    using vertex_id = CSRGraph::vertex_id;
    using count_type = CSRGraph::offset_type;

    struct VertexRange {
        vertex_id begin = 0;
        vertex_id end = 0;
    };

    struct PartitionActivity {
        count_type active_vertices = 0;
        count_type active_edges = 0;
        count_type total_edges = 0;
        [[nodiscard]] bool has_active_vertices() const noexcept { return active_vertices != 0U; }
        [[nodiscard]] bool has_active_edges() const noexcept { return active_edges != 0U; }
    };

    explicit ActivityTracker(count_type vertex_count);

    [[nodiscard]] count_type vertex_count() const noexcept { return vertex_count_; }
    void clear() noexcept;
    // Throws std::out_of_range for an unknown vertex.
    void set_active(vertex_id vertex, bool active = true);
    [[nodiscard]] bool is_active(vertex_id vertex) const;
    // Replaces the active set (duplicates are harmless).
    void set_active_vertices(const std::vector<vertex_id> &vertices);
    // Ascending vertex ids.
    [[nodiscard]] std::vector<vertex_id> active_vertices() const;
    [[nodiscard]] count_type active_vertex_count() const noexcept { return active_count_; }
    [[nodiscard]] count_type active_edge_count(const CSRGraph &graph) const;
    [[nodiscard]] std::vector<PartitionActivity> partition_statistics(
        const CSRGraph &graph, const std::vector<VertexRange> &partitions) const;

    // Raw byte-per-vertex flags (1 = active), for bulk upload to the device.
    [[nodiscard]] const std::vector<unsigned char> &flags() const noexcept { return active_; }

private:
    count_type vertex_count_ = 0;
    std::vector<unsigned char> active_;
    count_type active_count_ = 0;

    void check_vertex(vertex_id vertex) const;
    void check_graph(const CSRGraph &graph) const;
    void check_range(const VertexRange &range) const;
};

}  // namespace hytgraph::graph
