// pagerank_gpu / sssp_gpu: the reference's C++ GPU entry points
// (include/algorithms/pagerank.hpp:50-52, include/algorithms/sssp.hpp:49-51)
// as thin wrappers over the C ABI.  Input is validated on the host first
// with the reference's messages (src/algorithms/pagerank.cpp:62-85,
// src/algorithms/sssp.cpp:82-124) so the exception types match; CUDA-side
// failures surface as std::runtime_error("<entry>: <message>").
#include "algorithms/pagerank.hpp"
#include "algorithms/sssp.hpp"
#include "hyt/capi.h"

#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

namespace hytgraph::algorithms {
namespace {

void require_device(const char *entry) {
    int n = 0;
    if (hyt_device_count(&n) != HYT_OK || n == 0)
        throw std::runtime_error(std::string(entry) + ": no CUDA device is available");
}

void check(int status, const char *entry) {
    if (status == HYT_OK) return;
    const std::string msg = std::string(entry) + ": " + hyt_last_error();
    if (status == HYT_E_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// Owns a device graph for the duration of one call.
struct DeviceGraph {
    hyt_graph *g = nullptr;
    DeviceGraph(const graph::CSRGraph &graph, const void *weights, uint32_t kind, uint32_t flags, const char *entry) {
        hyt_csr csr{};
        csr.num_vertices = graph.num_vertices();
        csr.num_edges = graph.num_edges();
        csr.row_offsets = graph.row_offsets().data();
        csr.column_indices = graph.column_indices().data();
        csr.weights = weights;
        csr.weight_kind = kind;
        hyt_graph_options opt{};
        opt.flags = flags;
        opt.device = -1;  // the calling thread's current device, as the reference's solvers use
        check(hyt_graph_create(&csr, &opt, &g), entry);
    }
    ~DeviceGraph() {
        if (g) hyt_graph_destroy(g);
    }
    DeviceGraph(const DeviceGraph &) = delete;
    DeviceGraph &operator=(const DeviceGraph &) = delete;
};

void validate_sssp(const graph::CSRGraph &graph, const SSSPOptions &options) {
    if (graph.num_vertices() == 0U) throw std::invalid_argument("SSSP requires at least one vertex");
    if (static_cast<graph::CSRGraph::offset_type>(options.source) >= graph.num_vertices())
        throw std::invalid_argument("SSSP source vertex is out of range");
    if (!(options.tolerance >= 0.0F) || !std::isfinite(options.tolerance))
        throw std::invalid_argument("SSSP tolerance must be finite and non-negative");
    for (const float w : graph.edge_weights())
        if (!std::isfinite(w) || w < 0.0F) throw std::invalid_argument("SSSP requires finite non-negative edge weights");
    if (options.tolerance > 0.0F)
        throw std::invalid_argument("sssp_gpu: a positive tolerance is not supported by the exact GPU solver");
}

uint32_t rounds_limit(std::size_t max_iterations) {
    if (max_iterations == 0U) return 0U;
    return max_iterations > 0xFFFFFFF0ull ? 0xFFFFFFF0u : static_cast<uint32_t>(max_iterations);
}

}  // namespace

PageRankResult pagerank_gpu(const graph::CSRGraph &graph, const PageRankOptions &options) {
    if (graph.num_vertices() == 0U) throw std::invalid_argument("PageRank requires at least one vertex");
    if (!(options.damping_factor >= 0.0F && options.damping_factor < 1.0F))
        throw std::invalid_argument("PageRank damping_factor must be in [0, 1)");
    if (!(options.tolerance > 0.0F) || !std::isfinite(options.tolerance))
        throw std::invalid_argument("PageRank tolerance must be finite and positive");
    if (options.max_iterations == 0U) throw std::invalid_argument("PageRank max_iterations must be greater than zero");
    require_device("pagerank_gpu");

    DeviceGraph dg(graph, nullptr, HYT_WEIGHTS_NONE, HYT_GRAPH_PULL, "pagerank_gpu");
    hyt_pagerank_params p{};
    p.damping = options.damping_factor;
    p.tolerance = options.tolerance;
    p.max_iterations = options.max_iterations > 0xFFFFFFF0ull ? 0xFFFFFFF0u : static_cast<uint32_t>(options.max_iterations);
    PageRankResult r;
    r.ranks.resize(static_cast<std::size_t>(graph.num_vertices()));
    hyt_run_stats st{};
    check(hyt_pagerank(dg.g, &p, r.ranks.data(), &st), "pagerank_gpu");
    r.iterations = st.iterations;
    r.residual = static_cast<float>(st.residual);
    r.converged = st.converged != 0U;
    return r;
}

SSSPResult sssp_gpu(const graph::CSRGraph &graph, const SSSPOptions &options) {
    validate_sssp(graph, options);
    require_device("sssp_gpu");
    // Float weights relax with the same IEEE additions as the reference's
    // float solver, so distances match it bit for bit.
    const bool weighted = graph.has_weights();
    DeviceGraph dg(graph, weighted ? graph.edge_weights().data() : nullptr,
                   weighted ? HYT_WEIGHTS_F32 : HYT_WEIGHTS_NONE, HYT_GRAPH_PUSH, "sssp_gpu");
    hyt_sssp_params p{};
    p.source = options.source;
    p.max_rounds = rounds_limit(options.max_iterations);
    std::vector<uint32_t> raw(static_cast<std::size_t>(graph.num_vertices()));
    hyt_run_stats st{};
    check(hyt_sssp(dg.g, &p, raw.data(), &st), "sssp_gpu");
    SSSPResult r;
    r.distances.resize(raw.size());
    if (weighted) {
        std::memcpy(r.distances.data(), raw.data(), raw.size() * sizeof(float));
    } else {
        for (std::size_t i = 0; i < raw.size(); ++i)
            r.distances[i] = raw[i] == HYT_DIST_INF_U32 ? std::numeric_limits<float>::infinity()
                                                        : static_cast<float>(raw[i]);
    }
    r.iterations = st.iterations;
    r.converged = st.converged != 0U;
    return r;
}

SSSPResultU32 sssp_gpu_u32(const graph::CSRGraph &graph, const SSSPOptions &options) {
    validate_sssp(graph, options);
    std::vector<uint32_t> w;
    if (graph.has_weights()) {
        w.reserve(graph.edge_weights().size());
        for (const float x : graph.edge_weights()) {
            if (x != std::floor(x) || x > 4294967295.0F)
                throw std::invalid_argument("sssp_gpu_u32: weights must be integers below 2^32");
            w.push_back(static_cast<uint32_t>(x));
        }
    }
    require_device("sssp_gpu_u32");
    DeviceGraph dg(graph, w.empty() ? nullptr : w.data(), w.empty() ? HYT_WEIGHTS_NONE : HYT_WEIGHTS_U32,
                   HYT_GRAPH_PUSH, "sssp_gpu_u32");
    hyt_sssp_params p{};
    p.source = options.source;
    p.max_rounds = rounds_limit(options.max_iterations);
    SSSPResultU32 r;
    r.distances.resize(static_cast<std::size_t>(graph.num_vertices()));
    hyt_run_stats st{};
    check(hyt_sssp(dg.g, &p, r.distances.data(), &st), "sssp_gpu_u32");
    r.iterations = st.iterations;
    r.converged = st.converged != 0U;
    return r;
}

std::vector<PageRankContribution> pagerank_contributions_gpu(const graph::CSRGraph &graph,
                                                             const std::vector<float> &current_ranks,
                                                             const PageRankOptions &options) {
    if (graph.num_vertices() == 0U) throw std::invalid_argument("PageRank requires at least one vertex");
    if (!(options.damping_factor >= 0.0F && options.damping_factor < 1.0F))
        throw std::invalid_argument("PageRank damping_factor must be in [0, 1)");
    if (current_ranks.size() != graph.num_vertices())
        throw std::invalid_argument("PageRank current_ranks size must match graph vertex count");
    require_device("pagerank_contributions_gpu");
    DeviceGraph dg(graph, nullptr, HYT_WEIGHTS_NONE, HYT_GRAPH_PULL, "pagerank_contributions_gpu");
    std::vector<double> c(current_ranks.size());
    check(hyt_pagerank_contributions(dg.g, current_ranks.data(), options.damping_factor, c.data()),
          "pagerank_contributions_gpu");
    std::vector<PageRankContribution> out(c.size());
    for (std::size_t v = 0; v < c.size(); ++v) out[v] = {v, c[v]};
    return out;
}

std::vector<SSSPContribution> sssp_contributions_gpu(const std::vector<float> &current_distances,
                                                     const std::vector<float> &candidate_distances, float tolerance) {
    if (!(tolerance >= 0.0F) || !std::isfinite(tolerance))
        throw std::invalid_argument("SSSP contribution tolerance must be finite and non-negative");
    if (current_distances.size() != candidate_distances.size())
        throw std::invalid_argument("SSSP contribution distance vectors must have equal size");
    std::vector<SSSPContribution> out(current_distances.size());
    if (out.empty()) return out;
    require_device("sssp_contributions_gpu");
    std::vector<double> c(out.size());
    check(hyt_sssp_contributions(current_distances.data(), candidate_distances.data(), c.size(), tolerance, c.data()),
          "sssp_contributions_gpu");
    for (std::size_t v = 0; v < c.size(); ++v) out[v] = {v, c[v]};
    return out;
}

}  // namespace hytgraph::algorithms
