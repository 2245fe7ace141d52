#pragma once
// SSSP interface, source-compatible with the reference
// (include/algorithms/sssp.hpp:11-51).
//
// sssp_gpu is implemented by this library.  sssp_cpu and sssp_contributions
// are the reference's CPU routines (src/algorithms/sssp.cpp), declared here
// for source compatibility and provided by linking the reference's sources.

#include "graph/csr_graph.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::algorithms {

struct SSSPOptions {
    graph::CSRGraph::vertex_id source = 0;
    float tolerance = 0.0F;
    std::size_t max_iterations = 0;  // 0: no limit beyond |V| rounds
};

struct SSSPContribution {
    std::size_t vertex = 0U;
    double contribution = 0.0;
};

[[nodiscard]] std::vector<SSSPContribution> sssp_contributions(const std::vector<float> &current_distances,
                                                               const std::vector<float> &candidate_distances,
                                                               float tolerance = 0.0F);
// sssp_contributions on the GPU (hyt_sssp_contributions), bit for bit.
[[nodiscard]] std::vector<SSSPContribution> sssp_contributions_gpu(const std::vector<float> &current_distances,
                                                                   const std::vector<float> &candidate_distances,
                                                                   float tolerance = 0.0F);

struct SSSPResult {
    std::vector<float> distances;  // +inf for unreachable vertices
    std::size_t iterations = 0;    // frontier rounds of the GPU schedule
    bool converged = false;
};

SSSPResult sssp_cpu(const graph::CSRGraph &graph, const SSSPOptions &options = {});

// Frontier SSSP on the GPU with atomicMin relaxation.  Distances equal the
// reference's bit for bit (integer weights: exact uint32 arithmetic; other
// float weights: the same IEEE additions).  options.tolerance must be 0 on
// this path (a positive tolerance makes the result schedule-dependent) and
// is rejected otherwise; `iterations` counts this solver's rounds.
SSSPResult sssp_gpu(const graph::CSRGraph &graph, const SSSPOptions &options = {});

// Exact integer distances (UINT32_MAX = unreachable) for graphs whose
// weights are non-negative integers below 2^32.
struct SSSPResultU32 {
    std::vector<std::uint32_t> distances;
    std::size_t iterations = 0;
    bool converged = false;
};
SSSPResultU32 sssp_gpu_u32(const graph::CSRGraph &graph, const SSSPOptions &options = {});

}  // namespace hytgraph::algorithms
