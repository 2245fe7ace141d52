// Host graph containers: CSRGraph, ActivityTracker, LogicalPartition(er).
// Behaviour (validation rules, exception types) follows the reference's
// src/graph/csr_graph.cpp:11-283, src/graph/activity_tracker.cpp:9-190 and
// src/graph/partition.cpp:8-197.
#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"
#include "hyt/capi.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace hytgraph::graph {

// ------------------------------- CSRGraph -------------------------------

CSRGraph::CSRGraph(offset_type num_vertices, std::vector<offset_type> row_offsets,
                   std::vector<vertex_id> column_indices, std::vector<weight_type> edge_weights)
    : num_vertices_(num_vertices),
      row_offsets_(std::move(row_offsets)),
      column_indices_(std::move(column_indices)),
      edge_weights_(std::move(edge_weights)) {
    validate();
}

std::pair<CSRGraph::offset_type, CSRGraph::offset_type> CSRGraph::neighbor_range(vertex_id vertex) const {
    if (static_cast<offset_type>(vertex) >= num_vertices_)
        throw std::out_of_range("CSRGraph::neighbor_range: vertex ID is out of range");
    return {row_offsets_[vertex], row_offsets_[static_cast<std::size_t>(vertex) + 1]};
}

CSRGraph::offset_type CSRGraph::out_degree(vertex_id vertex) const {
    const auto r = neighbor_range(vertex);
    return r.second - r.first;
}

CSRGraph::vertex_id CSRGraph::neighbor_at(offset_type edge_index) const {
    if (edge_index >= num_edges()) throw std::out_of_range("CSRGraph::neighbor_at: edge index is out of range");
    return column_indices_[static_cast<std::size_t>(edge_index)];
}

CSRGraph::weight_type CSRGraph::weight_at(offset_type edge_index) const {
    if (!has_weights()) throw std::logic_error("CSRGraph::weight_at: graph does not contain edge weights");
    if (edge_index >= num_edges()) throw std::out_of_range("CSRGraph::weight_at: edge index is out of range");
    return edge_weights_[static_cast<std::size_t>(edge_index)];
}

void CSRGraph::validate() const {
    if (row_offsets_.size() != static_cast<std::size_t>(num_vertices_) + 1U)
        throw std::invalid_argument("CSRGraph::validate: row_offsets must contain num_vertices + 1 entries");
    // num_vertices == UINT64_MAX wraps the expected size to 0 above
    if (row_offsets_.empty()) throw std::invalid_argument("CSRGraph::validate: row_offsets must not be empty");
    if (row_offsets_.front() != 0) throw std::invalid_argument("CSRGraph::validate: first row offset must be zero");
    if (std::adjacent_find(row_offsets_.begin(), row_offsets_.end(),
                           [](offset_type a, offset_type b) { return b < a; }) != row_offsets_.end())
        throw std::invalid_argument("CSRGraph::validate: row offsets must be non-decreasing");
    if (row_offsets_.back() != num_edges())
        throw std::invalid_argument("CSRGraph::validate: terminal row offset must equal number of edges");
    for (const vertex_id d : column_indices_)
        if (static_cast<offset_type>(d) >= num_vertices_)
            throw std::invalid_argument("CSRGraph::validate: column index contains an invalid destination vertex ID");
    if (!edge_weights_.empty() && edge_weights_.size() != column_indices_.size())
        throw std::invalid_argument("CSRGraph::validate: edge_weights must contain exactly one weight per edge");
}

// Runs on the GPU (hyt_csr_reorder, the steps of the reference's
// src/graph/csr_graph.cpp:171-283); the reference's messages for a wrong
// size, an out-of-range id or a duplicate id come back as
// std::invalid_argument.
void CSRGraph::reorder_vertices(const std::vector<vertex_id> &vertex_order) {
    const std::size_t n = static_cast<std::size_t>(num_vertices_);
    if (vertex_order.size() != n)
        throw std::invalid_argument("CSRGraph::reorder_vertices: vertex_order must contain exactly one entry per vertex");
    int devices = 0;
    if (hyt_device_count(&devices) != HYT_OK || devices == 0)
        throw std::runtime_error("CSRGraph::reorder_vertices: no CUDA device is available");
    hyt_csr csr{};
    csr.num_vertices = num_vertices_;
    csr.num_edges = num_edges();
    csr.row_offsets = row_offsets_.data();
    csr.column_indices = column_indices_.data();
    csr.weights = has_weights() ? edge_weights_.data() : nullptr;
    csr.weight_kind = has_weights() ? HYT_WEIGHTS_F32 : HYT_WEIGHTS_NONE;
    hyt_csr_buffers out{};
    const int status = hyt_csr_reorder(&csr, vertex_order.data(), 0, &out, nullptr);
    if (status != HYT_OK) {
        const std::string msg = hyt_last_error();
        if (status == HYT_E_INVALID) throw std::invalid_argument(msg);
        throw std::runtime_error("CSRGraph::reorder_vertices: " + msg);
    }
    const std::size_t m = column_indices_.size();
    std::vector<offset_type> offs(out.row_offsets, out.row_offsets + n + 1);
    std::vector<vertex_id> cols(out.column_indices, out.column_indices + m);
    std::vector<weight_type> wts;
    if (has_weights()) {
        wts.resize(m);
        if (m) std::memcpy(wts.data(), out.weights, m * sizeof(weight_type));
    }
    hyt_csr_buffers_free(&out);
    row_offsets_ = std::move(offs);
    column_indices_ = std::move(cols);
    edge_weights_ = std::move(wts);
}

// ---------------------------- ActivityTracker ----------------------------

ActivityTracker::ActivityTracker(count_type vertex_count)
    : vertex_count_(vertex_count), active_(static_cast<std::size_t>(vertex_count), 0U) {}

void ActivityTracker::check_vertex(vertex_id vertex) const {
    if (static_cast<count_type>(vertex) >= vertex_count_) throw std::out_of_range("activity vertex is out of range");
}

void ActivityTracker::check_graph(const CSRGraph &graph) const {
    if (graph.num_vertices() != vertex_count_)
        throw std::invalid_argument("activity tracker vertex count does not match graph");
}

void ActivityTracker::check_range(const VertexRange &range) const {
    if (range.begin > range.end) throw std::invalid_argument("activity partition range has begin greater than end");
    if (static_cast<count_type>(range.end) > vertex_count_)
        throw std::out_of_range("activity partition range exceeds vertex count");
}

void ActivityTracker::clear() noexcept {
    std::fill(active_.begin(), active_.end(), 0U);
    active_count_ = 0;
}

void ActivityTracker::set_active(vertex_id vertex, bool active) {
    check_vertex(vertex);
    unsigned char &f = active_[vertex];
    if ((f != 0U) == active) return;
    f = active ? 1U : 0U;
    if (active)
        ++active_count_;
    else
        --active_count_;
}

bool ActivityTracker::is_active(vertex_id vertex) const {
    check_vertex(vertex);
    return active_[vertex] != 0U;
}

void ActivityTracker::set_active_vertices(const std::vector<vertex_id> &vertices) {
    clear();
    for (const vertex_id v : vertices) set_active(v, true);
}

std::vector<ActivityTracker::vertex_id> ActivityTracker::active_vertices() const {
    std::vector<vertex_id> out;
    out.reserve(static_cast<std::size_t>(active_count_));
    for (std::size_t v = 0; v < active_.size(); ++v)
        if (active_[v]) out.push_back(static_cast<vertex_id>(v));
    return out;
}

ActivityTracker::count_type ActivityTracker::active_edge_count(const CSRGraph &graph) const {
    check_graph(graph);
    const auto &off = graph.row_offsets();
    count_type total = 0;
    for (std::size_t v = 0; v < active_.size(); ++v)
        if (active_[v]) total += off[v + 1] - off[v];
    return total;
}

std::vector<ActivityTracker::PartitionActivity> ActivityTracker::partition_statistics(
    const CSRGraph &graph, const std::vector<VertexRange> &partitions) const {
    check_graph(graph);
    const auto &off = graph.row_offsets();
    std::vector<PartitionActivity> out;
    out.reserve(partitions.size());
    for (const VertexRange &r : partitions) {
        check_range(r);
        PartitionActivity a;
        a.total_edges = off[r.end] - off[r.begin];
        for (std::size_t v = r.begin; v < r.end; ++v) {
            if (!active_[v]) continue;
            ++a.active_vertices;
            a.active_edges += off[v + 1] - off[v];
        }
        out.push_back(a);
    }
    return out;
}

// --------------------------- LogicalPartition(er) -------------------------

LogicalPartition::LogicalPartition(vertex_id vertex_begin, vertex_id vertex_end, offset_type edge_begin,
                                   offset_type edge_end, byte_type target_bytes)
    : vertex_begin_(vertex_begin),
      vertex_end_(vertex_end),
      edge_begin_(edge_begin),
      edge_end_(edge_end),
      target_bytes_(target_bytes) {
    if (vertex_begin_ > vertex_end_)
        throw std::invalid_argument("LogicalPartition: vertex_begin must not exceed vertex_end");
    if (edge_begin_ > edge_end_) throw std::invalid_argument("LogicalPartition: edge_begin must not exceed edge_end");
    if (target_bytes_ == 0U) throw std::invalid_argument("LogicalPartition: target_bytes must be greater than zero");
}

LogicalPartitioner::LogicalPartitioner(byte_type partition_bytes) : partition_bytes_(partition_bytes) {
    if (partition_bytes_ == 0U)
        throw std::invalid_argument("LogicalPartitioner: partition_bytes must be greater than zero");
}

void LogicalPartitioner::check_graph(const CSRGraph &graph) const {
    if (graph.num_vertices() == 0U) return;
    if (graph.row_offsets().size() != static_cast<std::size_t>(graph.num_vertices()) + 1U)
        throw std::invalid_argument("LogicalPartitioner: invalid CSR row-offset count");
    if (graph.row_offsets().back() != graph.num_edges())
        throw std::invalid_argument("LogicalPartitioner: CSR terminal offset does not match the number of edges");
}

std::vector<LogicalPartition> LogicalPartitioner::partition(const CSRGraph &graph) const {
    check_graph(graph);
    std::vector<LogicalPartition> parts;
    const auto n = static_cast<vertex_id>(graph.num_vertices());
    if (n == 0U) return parts;
    const auto &off = graph.row_offsets();
    vertex_id begin = 0;
    for (vertex_id v = 1; v < n; ++v) {
        // bytes of destination ids if row v joined the open partition
        const byte_type bytes = static_cast<byte_type>(off[v + 1] - off[begin]) * sizeof(vertex_id);
        if (bytes > partition_bytes_) {
            parts.emplace_back(begin, v, off[begin], off[v], partition_bytes_);
            begin = v;
        }
    }
    parts.emplace_back(begin, n, off[begin], off[n], partition_bytes_);
    return parts;
}

std::vector<LogicalPartition> LogicalPartitioner::partition_by_vertices(const CSRGraph &graph,
                                                                       vertex_id vertices_per_partition) {
    if (vertices_per_partition == 0U)
        throw std::invalid_argument("LogicalPartitioner: vertices_per_partition must be greater than zero");
    std::vector<LogicalPartition> parts;
    const auto &off = graph.row_offsets();
    const std::uint64_t n = graph.num_vertices();
    for (std::uint64_t b = 0; b < n; b += vertices_per_partition) {
        const std::uint64_t e = std::min<std::uint64_t>(n, b + vertices_per_partition);
        const byte_type bytes = std::max<byte_type>(1, static_cast<byte_type>(off[e] - off[b]) * sizeof(vertex_id));
        parts.emplace_back(static_cast<vertex_id>(b), static_cast<vertex_id>(e), off[b], off[e], bytes);
    }
    return parts;
}

}  // namespace hytgraph::graph
