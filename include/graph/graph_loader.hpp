#pragma once
// Edge-list loading.  Source-compatible with hytgraph::graph::GraphLoader
// (reference include/graph/graph_loader.hpp, src/graph/graph_loader.cpp:39-179):
// one "source destination [weight]" record per line, '#' comments and blank
// lines skipped, parallel edges kept, file order kept within a source.
// The file is parsed by host threads and the CSR built on the GPU
// (hyt_load_edge_list); std::invalid_argument for a bad record (with the
// reference's message and line), std::runtime_error for a file that cannot
// be read or when no CUDA device is available.
//
// save_csr / load_csr (no counterpart in the reference) write and read
// this library's binary CSR file (hyt_csr_save / hyt_csr_load): checksummed,
// structure-checked, loaded on the GPU.

#include "graph/csr_graph.hpp"

#include <string>

namespace hytgraph::graph {

class GraphLoader {
public:
    [[nodiscard]] static CSRGraph load_edge_list(const std::string &path, CSRGraph::offset_type num_vertices,
                                                 bool weighted = false);
    static void save_csr(const CSRGraph &graph, const std::string &path);
    [[nodiscard]] static CSRGraph load_csr(const std::string &path);
};

}  // namespace hytgraph::graph
