#pragma once
// PageRank interface, source-compatible with the reference
// (include/algorithms/pagerank.hpp:11-52).
//
// pagerank_gpu is implemented by this library (libhytgraph.so over the
// sm_100a core, libhyt_core.so).  pagerank_cpu and pagerank_contributions
// are the reference's own CPU routines (src/algorithms/pagerank.cpp); they
// stay declared here so code that calls both keeps compiling, and are
// provided by linking the reference's CPU sources.

#include "graph/csr_graph.hpp"

#include <cstddef>
#include <vector>

namespace hytgraph::algorithms {

struct PageRankOptions {
    float damping_factor = 0.85F;
    float tolerance = 1.0e-6F;  // stop when the L1 change <= tolerance
    std::size_t max_iterations = 100;
};

struct PageRankContribution {
    std::size_t vertex = 0U;
    double contribution = 0.0;
};

struct PageRankResult {
    std::vector<float> ranks;
    std::size_t iterations = 0;
    float residual = 0.0F;
    bool converged = false;
};

PageRankResult pagerank_cpu(const graph::CSRGraph &graph, const PageRankOptions &options = {});

[[nodiscard]] std::vector<PageRankContribution> pagerank_contributions(const graph::CSRGraph &graph,
                                                                       const std::vector<float> &current_ranks,
                                                                       const PageRankOptions &options = {});

// Synchronous (Jacobi) PageRank on the GPU, pull over the CSC, same update
// and stopping rule as pagerank_cpu.  Throws std::invalid_argument for bad
// input (same messages as the CPU solver) and std::runtime_error for CUDA
// failures or when no device is present.
PageRankResult pagerank_gpu(const graph::CSRGraph &graph, const PageRankOptions &options = {});
// pagerank_contributions on the GPU (hyt_pagerank_contributions; sums in
// FP64, so values agree with the FP32 reference to its rounding).
[[nodiscard]] std::vector<PageRankContribution> pagerank_contributions_gpu(const graph::CSRGraph &graph,
                                                                           const std::vector<float> &current_ranks,
                                                                           const PageRankOptions &options = {});

}  // namespace hytgraph::algorithms
