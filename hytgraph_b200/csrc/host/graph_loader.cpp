// GraphLoader (reference src/graph/graph_loader.cpp:39-179) over the C ABI:
// hyt_load_edge_list, and the binary CSR file (hyt_csr_save / hyt_csr_load).
#include "graph/graph_loader.hpp"

#include "hyt/capi.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace hytgraph::graph {
namespace {

void require_device(const char *entry) {
    int n = 0;
    if (hyt_device_count(&n) != HYT_OK || n == 0)
        throw std::runtime_error(std::string(entry) + ": no CUDA device is available");
}

void check(int status) {
    if (status == HYT_OK) return;
    const std::string msg = hyt_last_error();
    if (status == HYT_E_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// Takes host buffers from the library into a CSRGraph (float weights).
CSRGraph take(hyt_csr_buffers &b) {
    const std::size_t V = static_cast<std::size_t>(b.num_vertices), E = static_cast<std::size_t>(b.num_edges);
    std::vector<CSRGraph::offset_type> off(b.row_offsets, b.row_offsets + V + 1);
    std::vector<CSRGraph::vertex_id> cols(b.column_indices, b.column_indices + E);
    std::vector<CSRGraph::weight_type> w;
    if (b.weights) {
        w.resize(E);
        if (E) std::memcpy(w.data(), b.weights, E * sizeof(float));
    }
    hyt_csr_buffers_free(&b);
    return CSRGraph(V, std::move(off), std::move(cols), std::move(w));
}

}  // namespace

CSRGraph GraphLoader::load_edge_list(const std::string &path, CSRGraph::offset_type num_vertices, bool weighted) {
    require_device("GraphLoader::load_edge_list");
    hyt_csr_buffers b{};
    check(hyt_load_edge_list(path.c_str(), num_vertices, weighted ? 1 : 0, 0, &b, nullptr));
    return take(b);
}

void GraphLoader::save_csr(const CSRGraph &graph, const std::string &path) {
    require_device("GraphLoader::save_csr");
    hyt_csr csr{};
    csr.num_vertices = graph.num_vertices();
    csr.num_edges = graph.num_edges();
    csr.row_offsets = graph.row_offsets().data();
    csr.column_indices = graph.column_indices().data();
    csr.weights = graph.has_weights() ? graph.edge_weights().data() : nullptr;
    csr.weight_kind = graph.has_weights() ? HYT_WEIGHTS_F32 : HYT_WEIGHTS_NONE;
    check(hyt_csr_save(path.c_str(), &csr));
}

CSRGraph GraphLoader::load_csr(const std::string &path) {
    require_device("GraphLoader::load_csr");
    hyt_csr_buffers b{};
    check(hyt_csr_load(path.c_str(), 0, &b, nullptr));
    if (b.weights && b.weight_kind != HYT_WEIGHTS_F32) {
        hyt_csr_buffers_free(&b);
        throw std::invalid_argument("GraphLoader::load_csr: the file holds integer weights; CSRGraph holds floats");
    }
    return take(b);
}

}  // namespace hytgraph::graph
