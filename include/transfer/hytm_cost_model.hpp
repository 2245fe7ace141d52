#pragma once
// HyTM transfer-engine cost model and selector.  Source-compatible with
// hytgraph::transfer::HyTMCostModel (reference
// include/transfer/hytm_cost_model.hpp:15-211); the arithmetic follows the
// paper's formulas (1)-(3) and Algorithm 1 exactly as the reference states
// them (src/transfer/hytm_cost_model.cpp:454-715), so decisions are
// identical for identical inputs.  The executing engine
// (transfer/hybrid_engine.hpp) feeds the same arithmetic with per-partition
// metrics computed on the GPU and with measured link parameters.

#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::transfer {

enum class TransferEngine { ExpTMFilter, ExpTMCompaction, ImpTMZeroCopy };

struct HyTMCostModelOptions {
    double alpha = 0.80;   // compaction must beat alpha * filter ...
    double beta = 0.40;    // ... and beta * zero-copy (strictly)
    double gamma = 0.625;  // zero-copy RTT mixing factor
    std::size_t request_payload_bytes = 128U;  // m
    std::size_t max_requests_per_tlp = 256U;   // MR
    double rtt = 1.0;                          // time of one saturated TLP
    double cpu_compaction_throughput_bytes_per_second = 1.0;
    std::size_t destination_entry_bytes = sizeof(graph::CSRGraph::vertex_id);  // d1
    std::size_t vertex_index_bytes = sizeof(graph::CSRGraph::offset_type);     // d2
    std::size_t alignment_bytes = 128U;
};

struct HyTMPartitionMetrics {
    std::size_t partition_index = 0U;
    graph::CSRGraph::vertex_id vertex_begin = 0U;
    graph::CSRGraph::vertex_id vertex_end = 0U;
    graph::CSRGraph::offset_type active_vertices = 0U;
    graph::CSRGraph::offset_type active_edges = 0U;
    graph::CSRGraph::offset_type total_edges = 0U;
    std::uint64_t filter_transfer_bytes = 0U;         // E_p * d1
    std::uint64_t compaction_bytes = 0U;              // A_e * d1 + A_v * d2
    std::uint64_t zero_copy_memory_requests = 0U;     // sum ceil(deg * d1 / m)
    std::uint64_t zero_copy_alignment_overhead = 0U;  // sum am(v)
    std::uint64_t zero_copy_total_requests = 0U;
};

struct HyTMPartitionCosts {
    HyTMPartitionMetrics metrics;
    double filter_cost = 0.0;
    double compaction_cost = 0.0;
    double zero_copy_cost = 0.0;
    double zero_copy_rtt = 0.0;
    TransferEngine selected_engine = TransferEngine::ExpTMFilter;
};

class HyTMCostModel {
public:
    // Throws std::invalid_argument for out-of-range options.
    explicit HyTMCostModel(HyTMCostModelOptions options = {});

    [[nodiscard]] const HyTMCostModelOptions &options() const noexcept { return options_; }

    [[nodiscard]] HyTMPartitionCosts evaluate_partition(const graph::CSRGraph &graph,
                                                        const graph::LogicalPartition &partition,
                                                        const graph::ActivityTracker &activity,
                                                        std::size_t partition_index = 0U) const;

    [[nodiscard]] std::vector<HyTMPartitionCosts> evaluate_partitions(
        const graph::CSRGraph &graph, const std::vector<graph::LogicalPartition> &partitions,
        const graph::ActivityTracker &activity) const;

    // Costs from already-collected metrics (the GPU engine's path).
    [[nodiscard]] HyTMPartitionCosts evaluate_metrics(const HyTMPartitionMetrics &metrics) const;

    // Algorithm 1: C if C < alpha*F and C < beta*Z; else F if F < Z; else Z.
    [[nodiscard]] static TransferEngine select_engine(double filter_cost, double compaction_cost,
                                                      double zero_copy_cost, double alpha, double beta);

private:
    HyTMCostModelOptions options_;
};

}  // namespace hytgraph::transfer
