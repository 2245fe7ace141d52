// HubSorter (reference src/scheduling/hub_sort.cpp:28-183) over the GPU
// entry point hyt_hub_sort.
#include "scheduling/hub_sort.hpp"

#include "hyt/capi.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace hytgraph::scheduling {

HubSorter::HubSorter(HubSortOptions options) : options_(options) {
    if (!std::isfinite(options_.hub_fraction) || options_.hub_fraction < 0.0 || options_.hub_fraction > 1.0)
        throw std::invalid_argument("HubSortOptions.hub_fraction must be finite and in [0, 1]");
}

HubSortResult HubSorter::sort(const graph::CSRGraph &graph) const {
    HubSortResult r;
    const std::size_t n = static_cast<std::size_t>(graph.num_vertices());
    if (n == 0U) return r;
    int devices = 0;
    if (hyt_device_count(&devices) != HYT_OK || devices == 0)
        throw std::runtime_error("HubSorter::sort: no CUDA device is available");
    hyt_csr csr{};
    csr.num_vertices = graph.num_vertices();
    csr.num_edges = graph.num_edges();
    csr.row_offsets = graph.row_offsets().data();
    csr.column_indices = graph.column_indices().data();
    csr.weight_kind = HYT_WEIGHTS_NONE;
    r.vertex_order.resize(n);
    r.scores.resize(n);
    uint64_t hubs = 0;
    const int status =
        hyt_hub_sort(&csr, options_.hub_fraction, r.vertex_order.data(), r.scores.data(), &hubs, nullptr);
    if (status != HYT_OK) {
        const std::string msg = std::string("HubSorter::sort: ") + hyt_last_error();
        if (status == HYT_E_INVALID) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }
    r.hub_count = static_cast<std::size_t>(hubs);
    return r;
}

}  // namespace hytgraph::scheduling
