#pragma once
// Hub-first vertex ordering.  Source-compatible with
// hytgraph::scheduling::HubSorter (reference
// include/scheduling/hub_sort.hpp:10-89, src/scheduling/hub_sort.cpp:28-183):
//   H(v) = Do(v) * Di(v) / (Do_max * Di_max)   (0 on an edgeless graph),
//   the top hub_fraction of vertices (round when V*fraction is within 1e-12
//   of an integer, else ceil) ranked by higher score then lower id, followed
//   by every other vertex in its original order.
// sort() runs on the GPU (hyt_hub_sort); scores equal the reference's
// long-double quotient bit for bit.  It throws std::runtime_error when no
// CUDA device is available.

#include "graph/csr_graph.hpp"

#include <cstddef>
#include <vector>

namespace hytgraph::scheduling {

struct HubSortResult {
    std::vector<graph::CSRGraph::vertex_id> vertex_order;  // new id -> old id
    std::vector<double> scores;                            // by original id
    std::size_t hub_count = 0U;
    [[nodiscard]] bool empty() const noexcept { return vertex_order.empty(); }
};

struct HubSortOptions {
    double hub_fraction = 0.08;
};

class HubSorter {
public:
    // Throws std::invalid_argument unless hub_fraction is finite and in [0, 1].
    explicit HubSorter(HubSortOptions options = {});
    [[nodiscard]] const HubSortOptions &options() const noexcept { return options_; }
    [[nodiscard]] HubSortResult sort(const graph::CSRGraph &graph) const;

private:
    HubSortOptions options_;
};

}  // namespace hytgraph::scheduling
