// Transfer-layer host logic: ExpTM-Filter plans, ExpTM-Compaction payloads,
// ImpTM-Zero-Copy request metrics and the HyTM cost model.
//
// Decisions and metrics match the reference (src/transfer/filter_engine.cpp:
// 146-220, compaction_engine.cpp:253-492, zero_copy_engine.cpp:231-393,
// hytm_cost_model.cpp:330-715); the cost arithmetic is one function
// (costs_from_metrics) shared with the GPU-driven engine, which supplies
// metrics computed on the device.
#include "transfer/compaction_engine.hpp"
#include "transfer/filter_engine.hpp"
#include "transfer/hytm_cost_model.hpp"
#include "transfer/zero_copy_engine.hpp"

#include <chrono>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

namespace hytgraph::transfer {
namespace {

using graph::CSRGraph;
using graph::LogicalPartition;
using VertexId = CSRGraph::vertex_id;
using Offset = CSRGraph::offset_type;

std::uint64_t ceil_div(std::uint64_t n, std::uint64_t d) { return n / d + (n % d != 0U ? 1U : 0U); }

std::uint64_t mul_checked(std::uint64_t a, std::uint64_t b, const char *what) {
    if (a != 0U && b > std::numeric_limits<std::uint64_t>::max() / a) throw std::overflow_error(what);
    return a * b;
}

std::uint64_t add_checked(std::uint64_t a, std::uint64_t b, const char *what) {
    if (b > std::numeric_limits<std::uint64_t>::max() - a) throw std::overflow_error(what);
    return a + b;
}

// Contiguous, complete coverage of vertices and edges (shared by Filter and
// Zero-Copy; Zero-Copy also requires CSR row boundaries).
void check_cover(const CSRGraph &g, const std::vector<LogicalPartition> &parts, bool row_aligned) {
    VertexId next_v = 0;
    Offset next_e = 0;
    for (const LogicalPartition &p : parts) {
        if (p.vertex_begin() != next_v) throw std::invalid_argument("logical partitions must cover vertices contiguously");
        if (p.edge_begin() != next_e) throw std::invalid_argument("logical partitions must cover edges contiguously");
        if (p.vertex_begin() > p.vertex_end()) throw std::invalid_argument("logical partition has invalid vertex range");
        if (p.edge_begin() > p.edge_end()) throw std::invalid_argument("logical partition has invalid edge range");
        if (static_cast<Offset>(p.vertex_end()) > g.num_vertices())
            throw std::out_of_range("logical partition vertex range exceeds graph");
        if (p.edge_end() > g.num_edges()) throw std::out_of_range("logical partition edge range exceeds graph");
        if (row_aligned) {
            if (g.row_offsets()[p.vertex_begin()] != p.edge_begin())
                throw std::invalid_argument("logical partition edge_begin is not a CSR row boundary");
            if (g.row_offsets()[p.vertex_end()] != p.edge_end())
                throw std::invalid_argument("logical partition edge_end is not a CSR row boundary");
        }
        next_v = p.vertex_end();
        next_e = p.edge_end();
    }
    if (next_v != g.num_vertices()) throw std::invalid_argument("logical partitions do not cover all graph vertices");
    if (next_e != g.num_edges()) throw std::invalid_argument("logical partitions do not cover all graph edges");
}

std::vector<graph::ActivityTracker::VertexRange> ranges_of(const std::vector<LogicalPartition> &parts) {
    std::vector<graph::ActivityTracker::VertexRange> r;
    r.reserve(parts.size());
    for (const auto &p : parts) r.push_back({p.vertex_begin(), p.vertex_end()});
    return r;
}

void check_cost_options(const HyTMCostModelOptions &o) {
    if (!std::isfinite(o.alpha) || !std::isfinite(o.beta) || !std::isfinite(o.gamma))
        throw std::invalid_argument("HyTMCostModel: alpha, beta, and gamma must be finite");
    if (o.alpha <= 0.0) throw std::invalid_argument("HyTMCostModel: alpha must be greater than zero");
    if (o.beta <= 0.0) throw std::invalid_argument("HyTMCostModel: beta must be greater than zero");
    if (o.gamma < 0.0 || o.gamma > 1.0) throw std::invalid_argument("HyTMCostModel: gamma must be in the range [0, 1]");
    if (!std::isfinite(o.rtt) || o.rtt < 0.0)
        throw std::invalid_argument("HyTMCostModel: RTT must be finite and non-negative");
    if (!std::isfinite(o.cpu_compaction_throughput_bytes_per_second) ||
        o.cpu_compaction_throughput_bytes_per_second <= 0.0)
        throw std::invalid_argument("HyTMCostModel: CPU compaction throughput must be finite and greater than zero");
    if (o.request_payload_bytes == 0U)
        throw std::invalid_argument("HyTMCostModel: request payload size must be greater than zero");
    if (o.max_requests_per_tlp == 0U)
        throw std::invalid_argument("HyTMCostModel: maximum requests per TLP must be greater than zero");
    if (o.destination_entry_bytes == 0U)
        throw std::invalid_argument("HyTMCostModel: destination entry size must be greater than zero");
    if (o.vertex_index_bytes == 0U)
        throw std::invalid_argument("HyTMCostModel: vertex index size must be greater than zero");
    if (o.alignment_bytes == 0U) throw std::invalid_argument("HyTMCostModel: alignment size must be greater than zero");
}

}  // namespace

// ------------------------------- Filter ---------------------------------

std::size_t FilterTransferPlan::active_partition_count() const noexcept {
    std::size_t n = 0;
    for (const auto &p : partitions) n += p.active ? 1U : 0U;
    return n;
}
std::size_t FilterTransferPlan::transferred_partition_count() const noexcept {
    std::size_t n = 0;
    for (const auto &p : partitions) n += p.transferred ? 1U : 0U;
    return n;
}
CSRGraph::offset_type FilterTransferPlan::transferred_edge_count() const noexcept {
    CSRGraph::offset_type n = 0;
    for (const auto &p : partitions) n += p.transferred_edges;
    return n;
}
std::size_t FilterTransferPlan::transferred_byte_count() const noexcept {
    std::size_t n = 0;
    for (const auto &p : partitions) n += p.transferred_bytes;
    return n;
}

FilterTransferPlan ExpTMFilter::plan(const CSRGraph &graph, const std::vector<LogicalPartition> &partitions,
                                     const graph::ActivityTracker &activity) const {
    if (activity.vertex_count() != graph.num_vertices())
        throw std::invalid_argument("activity tracker vertex count does not match graph");
    check_cover(graph, partitions, false);
    const auto stats = activity.partition_statistics(graph, ranges_of(partitions));
    FilterTransferPlan plan;
    plan.partitions.reserve(partitions.size());
    for (std::size_t i = 0; i < partitions.size(); ++i) {
        FilterPartitionDecision d;
        d.partition_index = i;
        d.active = stats[i].active_edges != 0U;
        d.active_edges = stats[i].active_edges;
        d.total_edges = partitions[i].edge_count();
        d.transferred = !enabled_ || d.active;
        if (d.transferred) {
            d.transferred_edges = partitions[i].edge_count();
            d.transferred_bytes = partitions[i].edge_data_bytes();
        }
        plan.partitions.push_back(d);
    }
    return plan;
}

// ------------------------------ Compaction ------------------------------

CSRGraph::offset_type CompactedPartition::active_edge_count() const noexcept {
    return static_cast<CSRGraph::offset_type>(neighbors.size());
}

CSRGraph::offset_type CompactionResult::active_edge_count() const noexcept {
    CSRGraph::offset_type n = 0;
    for (const auto &p : partitions) n += p.active_edge_count();
    return n;
}
CSRGraph::offset_type CompactionResult::active_vertex_count() const noexcept {
    CSRGraph::offset_type n = 0;
    for (const auto &p : partitions) n += p.active_vertex_count();
    return n;
}
std::size_t CompactionResult::neighbor_bytes() const noexcept {
    std::size_t n = 0;
    for (const auto &p : partitions) n += p.neighbor_bytes();
    return n;
}
std::size_t CompactionResult::index_bytes() const noexcept {
    std::size_t n = 0;
    for (const auto &p : partitions) n += p.index_bytes();
    return n;
}
std::size_t CompactionResult::total_bytes() const noexcept { return neighbor_bytes() + index_bytes(); }

CompactionResult ExpTMCompaction::compact(const CSRGraph &graph, const std::vector<LogicalPartition> &partitions,
                                          const graph::ActivityTracker &activity) const {
    CompactionResult result;
    if (!enabled_) return result;
    if (activity.vertex_count() != graph.num_vertices())
        throw std::invalid_argument("ExpTMCompaction: activity tracker vertex count does not match graph");
    const auto t0 = std::chrono::steady_clock::now();
    const auto &off = graph.row_offsets();
    const auto &cols = graph.column_indices();
    const auto &flags = activity.flags();
    const auto nv = static_cast<VertexId>(graph.num_vertices());
    for (std::size_t pi = 0; pi < partitions.size(); ++pi) {
        const LogicalPartition &p = partitions[pi];
        if (p.vertex_begin() > p.vertex_end()) throw std::invalid_argument("ExpTMCompaction: partition vertex range is invalid");
        if (p.vertex_end() > nv) throw std::invalid_argument("ExpTMCompaction: partition vertex range exceeds graph");
        if (p.edge_begin() > p.edge_end()) throw std::invalid_argument("ExpTMCompaction: partition edge range is invalid");
        if (p.edge_end() > graph.num_edges()) throw std::invalid_argument("ExpTMCompaction: partition edge range exceeds graph");
        if (p.vertex_begin() < nv && off[p.vertex_begin()] != p.edge_begin())
            throw std::invalid_argument("ExpTMCompaction: partition edge_begin does not match its first CSR row");
        if (p.vertex_end() > p.vertex_begin() && off[p.vertex_end()] != p.edge_end())
            throw std::invalid_argument("ExpTMCompaction: partition edge_end does not match its final CSR row");
        CompactedPartition c;
        c.partition_index = pi;
        c.vertex_begin = p.vertex_begin();
        c.vertex_end = p.vertex_end();
        Offset payload = 0;
        for (VertexId v = p.vertex_begin(); v < p.vertex_end(); ++v) {
            if (!flags[v]) continue;
            c.active_vertices.push_back(v);
            payload += off[v + 1] - off[v];
        }
        if (c.active_vertices.empty()) continue;  // inactive partitions ship nothing
        c.neighbors.reserve(static_cast<std::size_t>(payload));
        c.neighbor_index.reserve(c.active_vertices.size() + 1);
        c.neighbor_index.push_back(0);
        for (const VertexId v : c.active_vertices) {
            c.neighbors.insert(c.neighbors.end(), cols.begin() + static_cast<std::ptrdiff_t>(off[v]),
                               cols.begin() + static_cast<std::ptrdiff_t>(off[v + 1]));
            c.neighbor_index.push_back(static_cast<Offset>(c.neighbors.size()));
        }
        result.partitions.push_back(std::move(c));
    }
    result.compaction_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return result;
}

std::vector<CSRGraph::vertex_id> ExpTMCompaction::expanded_neighbors(const CompactedPartition &p) {
    if (p.neighbor_index.size() != p.active_vertices.size() + 1U)
        throw std::invalid_argument(
            "ExpTMCompaction::expanded_neighbors: compressed index size does not match active vertex count");
    if (p.neighbor_index.front() != 0U)
        throw std::invalid_argument("ExpTMCompaction::expanded_neighbors: index must start at zero");
    if (p.neighbor_index.back() != static_cast<Offset>(p.neighbors.size()))
        throw std::invalid_argument("ExpTMCompaction::expanded_neighbors: terminal index does not match neighbor count");
    for (std::size_t i = 1; i < p.neighbor_index.size(); ++i)
        if (p.neighbor_index[i] < p.neighbor_index[i - 1])
            throw std::invalid_argument("ExpTMCompaction::expanded_neighbors: index is not monotonic");
    return p.neighbors;
}

// ------------------------------ Zero-copy -------------------------------

ZeroCopyResult ImpTMZeroCopy::prepare(const CSRGraph &graph, const std::vector<LogicalPartition> &partitions,
                                      const graph::ActivityTracker &activity) const {
    const auto t0 = std::chrono::steady_clock::now();
    if (options_.request_payload_bytes == 0U)
        throw std::invalid_argument("zero-copy request payload size must be greater than zero");
    if (options_.max_requests_per_tlp == 0U)
        throw std::invalid_argument("zero-copy maximum requests per TLP must be greater than zero");
    if (options_.alignment_bytes == 0U) throw std::invalid_argument("zero-copy alignment size must be greater than zero");
    if (activity.vertex_count() != graph.num_vertices())
        throw std::invalid_argument("activity tracker vertex count does not match graph");
    check_cover(graph, partitions, true);

    ZeroCopyResult r;
    r.mode = ZeroCopyMode::Modeled;  // metrics only; mapped reads happen in the hybrid engine
    r.host_memory_mapped = false;
    const auto &off = graph.row_offsets();
    const auto &flags = activity.flags();
    const std::uint64_t m = options_.request_payload_bytes, align = options_.alignment_bytes;
    r.partitions.reserve(partitions.size());
    for (std::size_t i = 0; i < partitions.size(); ++i) {
        const LogicalPartition &p = partitions[i];
        ZeroCopyPartition z;
        z.partition_index = i;
        z.vertex_begin = p.vertex_begin();
        z.vertex_end = p.vertex_end();
        for (VertexId v = p.vertex_begin(); v < p.vertex_end(); ++v) {
            if (!flags[v]) continue;
            ZeroCopyVertexMetrics vm;
            vm.vertex = v;
            vm.degree = off[v + 1] - off[v];
            vm.memory_requests = ceil_div(mul_checked(vm.degree, sizeof(VertexId), "zero-copy byte count overflow"), m);
            const std::uint64_t start = mul_checked(off[v], sizeof(VertexId), "zero-copy logical neighbor byte offset overflow");
            vm.alignment_overhead = (vm.degree != 0U && start % align != 0U) ? 1U : 0U;
            z.active_vertices.push_back(v);
            z.active_edge_count += vm.degree;
            z.memory_request_count += vm.memory_requests;
            z.alignment_overhead_count += vm.alignment_overhead;
            z.vertex_metrics.push_back(vm);
        }
        // The reference leaves the per-partition TLP count at 0 and only
        // reports the global one (zero_copy_engine.cpp:351-356, 384-388).
        z.modeled_tlp_count = 0;
        if (!z.active_vertices.empty()) ++r.active_partition_count;
        r.active_vertex_count += z.active_vertices.size();
        r.active_edge_count += z.active_edge_count;
        r.memory_request_count += z.memory_request_count;
        r.alignment_overhead_count += z.alignment_overhead_count;
        r.partitions.push_back(std::move(z));
    }
    r.modeled_tlp_count = ceil_div(r.memory_request_count, options_.max_requests_per_tlp);
    r.preparation_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return r;
}

// ------------------------------ Cost model ------------------------------

HyTMCostModel::HyTMCostModel(HyTMCostModelOptions options) : options_(options) { check_cost_options(options_); }

HyTMPartitionCosts HyTMCostModel::evaluate_metrics(const HyTMPartitionMetrics &metrics) const {
    check_cost_options(options_);
    const HyTMCostModelOptions &o = options_;
    HyTMPartitionCosts c;
    c.metrics = metrics;
    const std::uint64_t tlp_bytes = mul_checked(o.request_payload_bytes, o.max_requests_per_tlp,
                                                "HyTMCostModel: TLP byte capacity overflow");
    // (1) Filter: ceil(E_p d1 / (m MR)) * RTT
    c.filter_cost = static_cast<double>(ceil_div(metrics.filter_transfer_bytes, tlp_bytes)) * o.rtt;
    // (2) Compaction: ceil((A_e d1 + A_v d2) / (m MR)) * RTT + bytes / T_cpu
    c.compaction_cost = static_cast<double>(ceil_div(metrics.compaction_bytes, tlp_bytes)) * o.rtt +
                        static_cast<double>(metrics.compaction_bytes) / o.cpu_compaction_throughput_bytes_per_second;
    // (3) Zero-copy: ceil(sum(ceil(deg d1 / m) + am) / MR) * RTT_zc,
    //     RTT_zc = gamma RTT + (1 - gamma) (A_e / E_p) RTT
    c.zero_copy_rtt = metrics.total_edges == 0U
                          ? o.gamma * o.rtt
                          : o.gamma * o.rtt + (1.0 - o.gamma) *
                                                  (static_cast<double>(metrics.active_edges) /
                                                   static_cast<double>(metrics.total_edges)) *
                                                  o.rtt;
    c.zero_copy_cost =
        static_cast<double>(ceil_div(metrics.zero_copy_total_requests, o.max_requests_per_tlp)) * c.zero_copy_rtt;
    c.selected_engine = select_engine(c.filter_cost, c.compaction_cost, c.zero_copy_cost, o.alpha, o.beta);
    return c;
}

HyTMPartitionCosts HyTMCostModel::evaluate_partition(const CSRGraph &graph, const LogicalPartition &partition,
                                                     const graph::ActivityTracker &activity,
                                                     std::size_t partition_index) const {
    check_cost_options(options_);
    if (activity.vertex_count() != graph.num_vertices())
        throw std::invalid_argument("HyTMCostModel: activity tracker vertex count does not match graph");
    const auto &off = graph.row_offsets();
    if (partition.vertex_begin() > partition.vertex_end())
        throw std::invalid_argument("HyTMCostModel: partition vertex range is invalid");
    if (static_cast<Offset>(partition.vertex_end()) > graph.num_vertices())
        throw std::invalid_argument("HyTMCostModel: partition vertex range exceeds graph");
    if (partition.edge_begin() > partition.edge_end())
        throw std::invalid_argument("HyTMCostModel: partition edge range is invalid");
    if (partition.edge_end() > graph.num_edges())
        throw std::invalid_argument("HyTMCostModel: partition edge range exceeds graph");
    if (off[partition.vertex_begin()] != partition.edge_begin())
        throw std::invalid_argument("HyTMCostModel: partition edge_begin does not match its CSR row boundary");
    if (off[partition.vertex_end()] != partition.edge_end())
        throw std::invalid_argument("HyTMCostModel: partition edge_end does not match its CSR row boundary");

    const HyTMCostModelOptions &o = options_;
    HyTMPartitionMetrics m;
    m.partition_index = partition_index;
    m.vertex_begin = partition.vertex_begin();
    m.vertex_end = partition.vertex_end();
    m.total_edges = partition.edge_count();
    m.filter_transfer_bytes = mul_checked(m.total_edges, o.destination_entry_bytes,
                                          "HyTMCostModel: filter transfer byte count overflow");
    const auto &flags = activity.flags();
    for (VertexId v = partition.vertex_begin(); v < partition.vertex_end(); ++v) {
        if (!flags[v]) continue;
        ++m.active_vertices;
        const Offset deg = off[v + 1] - off[v];
        m.active_edges = add_checked(m.active_edges, deg, "HyTMCostModel: active edge count overflow");
        if (deg == 0U) continue;
        const std::uint64_t bytes = mul_checked(deg, o.destination_entry_bytes,
                                                "HyTMCostModel: zero-copy vertex byte count overflow");
        m.zero_copy_memory_requests = add_checked(m.zero_copy_memory_requests, ceil_div(bytes, o.request_payload_bytes),
                                                  "HyTMCostModel: zero-copy request count overflow");
        const std::uint64_t start = mul_checked(off[v], o.destination_entry_bytes,
                                                "HyTMCostModel: logical neighbor byte offset overflow");
        if (start % o.alignment_bytes != 0U) ++m.zero_copy_alignment_overhead;
    }
    m.compaction_bytes = add_checked(
        mul_checked(m.active_edges, o.destination_entry_bytes, "HyTMCostModel: compaction edge byte count overflow"),
        mul_checked(m.active_vertices, o.vertex_index_bytes, "HyTMCostModel: compaction index byte count overflow"),
        "HyTMCostModel: compaction transfer byte count overflow");
    m.zero_copy_total_requests = add_checked(m.zero_copy_memory_requests, m.zero_copy_alignment_overhead,
                                             "HyTMCostModel: zero-copy total request count overflow");
    return evaluate_metrics(m);
}

std::vector<HyTMPartitionCosts> HyTMCostModel::evaluate_partitions(const CSRGraph &graph,
                                                                   const std::vector<LogicalPartition> &partitions,
                                                                   const graph::ActivityTracker &activity) const {
    check_cost_options(options_);
    if (activity.vertex_count() != graph.num_vertices())
        throw std::invalid_argument("HyTMCostModel: activity tracker vertex count does not match graph");
    std::vector<HyTMPartitionCosts> out;
    out.reserve(partitions.size());
    for (std::size_t i = 0; i < partitions.size(); ++i) out.push_back(evaluate_partition(graph, partitions[i], activity, i));
    return out;
}

TransferEngine HyTMCostModel::select_engine(double filter_cost, double compaction_cost, double zero_copy_cost,
                                            double alpha, double beta) {
    if (!std::isfinite(filter_cost) || !std::isfinite(compaction_cost) || !std::isfinite(zero_copy_cost))
        throw std::invalid_argument("HyTMCostModel::select_engine: costs must be finite");
    if (filter_cost < 0.0 || compaction_cost < 0.0 || zero_copy_cost < 0.0)
        throw std::invalid_argument("HyTMCostModel::select_engine: costs must be non-negative");
    if (!std::isfinite(alpha) || alpha <= 0.0)
        throw std::invalid_argument("HyTMCostModel::select_engine: alpha must be finite and greater than zero");
    if (!std::isfinite(beta) || beta <= 0.0)
        throw std::invalid_argument("HyTMCostModel::select_engine: beta must be finite and greater than zero");
    if (compaction_cost < alpha * filter_cost && compaction_cost < beta * zero_copy_cost)
        return TransferEngine::ExpTMCompaction;
    if (filter_cost < zero_copy_cost) return TransferEngine::ExpTMFilter;
    return TransferEngine::ImpTMZeroCopy;
}

}  // namespace hytgraph::transfer
