#pragma once
// Host CSR graph.  Source-compatible with hytgraph::graph::CSRGraph
// (reference include/graph/csr_graph.hpp:11-69): uint32 vertex ids, uint64
// row offsets, optional float weights.  The device copy lives behind the
// C ABI (hyt/capi.h, hyt_graph_create).

#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>

namespace hytgraph::graph {

class CSRGraph {
public:
    using vertex_id = std::uint32_t;
    using offset_type = std::uint64_t;
    using weight_type = float;

    CSRGraph() = default;
    // Validates on construction; throws std::invalid_argument if malformed.
    CSRGraph(offset_type num_vertices, std::vector<offset_type> row_offsets,
             std::vector<vertex_id> column_indices, std::vector<weight_type> edge_weights = {});

    [[nodiscard]] offset_type num_vertices() const noexcept { return num_vertices_; }
    [[nodiscard]] offset_type num_edges() const noexcept { return static_cast<offset_type>(column_indices_.size()); }
    [[nodiscard]] bool has_weights() const noexcept { return !edge_weights_.empty(); }

    // Out-edges of `vertex`; throws std::out_of_range for an unknown vertex.
    [[nodiscard]] offset_type out_degree(vertex_id vertex) const;
    // [begin, end) into column_indices(); throws std::out_of_range.
    [[nodiscard]] std::pair<offset_type, offset_type> neighbor_range(vertex_id vertex) const;
    [[nodiscard]] vertex_id neighbor_at(offset_type edge_index) const;
    // Throws std::logic_error on an unweighted graph.
    [[nodiscard]] weight_type weight_at(offset_type edge_index) const;

    [[nodiscard]] const std::vector<offset_type> &row_offsets() const noexcept { return row_offsets_; }
    [[nodiscard]] const std::vector<vertex_id> &column_indices() const noexcept { return column_indices_; }
    [[nodiscard]] const std::vector<weight_type> &edge_weights() const noexcept { return edge_weights_; }

    // Throws std::invalid_argument when an invariant does not hold.
    void validate() const;

    // vertex_order[new_id] = old_id; adjacency lists follow their vertex and
    // destinations are renumbered.
    void reorder_vertices(const std::vector<vertex_id> &vertex_order);

private:
    offset_type num_vertices_ = 0;
    std::vector<offset_type> row_offsets_;
    std::vector<vertex_id> column_indices_;
    std::vector<weight_type> edge_weights_;
};

}  // namespace hytgraph::graph
