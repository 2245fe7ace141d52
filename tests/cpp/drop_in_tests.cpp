// Drop-in tests: code written against the reference's C++ interfaces
// (include/graph, include/algorithms, include/transfer, include/scheduling,
// include/runtime) compiled and linked against libhytgraph.so.
//
//   drop_in_tests cpu   -- host-side classes (no GPU needed)
//   drop_in_tests gpu   -- pagerank_gpu / sssp_gpu (exit 77 without a device)
//
// Known answers come from the reference's own tests
// (tests/algorithm_tests.cpp:22-206, tests/cuda_algorithm_tests.cu:23-87,
// tests/unit_tests.cpp:2058-2466); the other cases are this project's.
#include "algorithms/pagerank.hpp"
#include "algorithms/sssp.hpp"
#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/graph_loader.hpp"
#include "graph/partition.hpp"
#include "hyt/capi.h"
#include "runtime/config.hpp"
#include "runtime/result.hpp"
#include "scheduling/contribution_scheduler.hpp"
#include "scheduling/hub_sort.hpp"
#include "scheduling/task_combiner.hpp"
#include "transfer/compaction_engine.hpp"
#include "transfer/filter_engine.hpp"
#include "transfer/hytm_cost_model.hpp"
#include "transfer/zero_copy_engine.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <unistd.h>
#include <functional>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

using namespace hytgraph;
using graph::ActivityTracker;
using graph::CSRGraph;
using graph::LogicalPartition;
using transfer::TransferEngine;

namespace {

int g_checks = 0;

void check(bool ok, const std::string &what) {
    ++g_checks;
    if (!ok) throw std::runtime_error("check failed: " + what);
}

template <class Ex, class F>
void throws(F &&f, const std::string &what) {
    bool got = false;
    try {
        f();
    } catch (const Ex &) {
        got = true;
    } catch (const std::exception &e) {
        throw std::runtime_error("wrong exception for " + what + ": " + e.what());
    }
    check(got, "throws: " + what);
}

bool close(double a, double b, double tol = 1e-12) { return std::fabs(a - b) <= tol; }

// 0->1, 0->2, 1->2, 2->0, 3 isolated
CSRGraph small_graph() { return CSRGraph(4, {0, 2, 3, 4, 4}, {1, 2, 2, 0}); }

// ------------------------------- graph ----------------------------------
void test_csr() {
    const CSRGraph g = small_graph();
    check(g.num_vertices() == 4 && g.num_edges() == 4 && !g.has_weights(), "csr sizes");
    check(g.out_degree(0) == 2 && g.out_degree(3) == 0, "out degree");
    check(g.neighbor_range(1) == std::make_pair<CSRGraph::offset_type, CSRGraph::offset_type>(2, 3), "range");
    check(g.neighbor_at(3) == 0, "neighbor_at");
    throws<std::out_of_range>([&] { (void)g.out_degree(4); }, "vertex out of range");
    throws<std::out_of_range>([&] { (void)g.neighbor_at(4); }, "edge out of range");
    throws<std::logic_error>([&] { (void)g.weight_at(0); }, "weight of unweighted graph");
    throws<std::invalid_argument>([] { CSRGraph(2, {0, 1}, {0}); }, "offset count");
    throws<std::invalid_argument>([] { CSRGraph(2, {1, 1, 1}, {0}); }, "first offset");
    throws<std::invalid_argument>([] { CSRGraph(2, {0, 2, 1}, {0, 1}); }, "monotone offsets");
    throws<std::invalid_argument>([] { CSRGraph(2, {0, 1, 2}, {0, 2}); }, "destination range");
    throws<std::invalid_argument>([] { CSRGraph(2, {0, 1, 2}, {0, 1}, {1.0F}); }, "weight count");
    CSRGraph w(3, {0, 2, 3, 3}, {1, 2, 2}, {5.F, 6.F, 7.F});
    throws<std::invalid_argument>([&] { w.reorder_vertices({0, 1}); }, "order size");  // checked before the GPU
}

void test_activity() {
    const CSRGraph g = small_graph();
    ActivityTracker a(4);
    a.set_active(0);
    a.set_active(0);
    a.set_active(2);
    check(a.active_vertex_count() == 2 && a.is_active(2) && !a.is_active(1), "activity flags");
    check(a.active_edge_count(g) == 3, "active edges = out-edges of active vertices");
    check(a.active_vertices() == std::vector<CSRGraph::vertex_id>({0, 2}), "ascending ids");
    const auto st = a.partition_statistics(g, {{0, 2}, {2, 4}});
    check(st[0].active_vertices == 1 && st[0].active_edges == 2 && st[0].total_edges == 3, "stats 0");
    check(st[1].active_vertices == 1 && st[1].active_edges == 1 && st[1].total_edges == 1, "stats 1");
    a.set_active(2, false);
    check(a.active_vertex_count() == 1, "deactivate");
    a.set_active_vertices({3, 1, 3});
    check(a.active_vertex_count() == 2 && !a.is_active(0), "replace set");
    throws<std::out_of_range>([&] { a.set_active(4); }, "activity vertex range");
    throws<std::invalid_argument>([&] { (void)a.partition_statistics(g, {{2, 1}}); }, "range order");
    throws<std::out_of_range>([&] { (void)a.partition_statistics(g, {{0, 5}}); }, "range end");
    ActivityTracker b(3);
    throws<std::invalid_argument>([&] { (void)b.active_edge_count(g); }, "graph mismatch");
}

void test_partitioner() {
    // degrees 3, 0, 5, 1, 2 -> 11 edges; 4-byte ids
    std::vector<CSRGraph::vertex_id> cols = {1, 2, 3, 0, 1, 3, 4, 0, 2, 0, 1};
    const CSRGraph g(5, {0, 3, 3, 8, 9, 11}, cols);
    const auto parts = graph::LogicalPartitioner(16).partition(g);  // 4 edges per partition
    std::vector<std::pair<uint32_t, uint32_t>> want = {{0, 2}, {2, 3}, {3, 5}};
    check(parts.size() == want.size(), "partition count");
    for (std::size_t i = 0; i < parts.size(); ++i) {
        check(parts[i].vertex_begin() == want[i].first && parts[i].vertex_end() == want[i].second, "bounds");
        check(parts[i].edge_begin() == g.row_offsets()[want[i].first], "edge begin");
        check(parts[i].edge_end() == g.row_offsets()[want[i].second], "edge end");
    }
    check(parts[1].edge_count() == 5 && parts[1].edge_data_bytes() == 20, "oversized single row kept whole");
    check(graph::LogicalPartitioner().partition(CSRGraph(0, {0}, {})).empty(), "empty graph");
    throws<std::invalid_argument>([] { graph::LogicalPartitioner(0); }, "zero target");
    throws<std::invalid_argument>([] { LogicalPartition(2, 1, 0, 0, 1); }, "partition order");
    const auto by = graph::LogicalPartitioner::partition_by_vertices(g, 2);
    check(by.size() == 3 && by[2].vertex_begin() == 4 && by[2].edge_count() == 2, "by vertices");
}

// ------------------------------- transfer -------------------------------
void test_filter() {
    const CSRGraph g = small_graph();
    const std::vector<LogicalPartition> parts = {{0, 1, 0, 2, 64}, {1, 3, 2, 4, 64}, {3, 4, 4, 4, 64}};
    ActivityTracker a(4);
    a.set_active(1);
    a.set_active(3);
    const auto plan = transfer::ExpTMFilter(true).plan(g, parts, a);
    check(plan.partitions.size() == 3, "filter size");
    check(!plan.partitions[0].transferred && plan.partitions[1].transferred && !plan.partitions[2].transferred,
          "filter skips partitions without active edges (vertex 3 has none)");
    check(plan.partitions[1].transferred_edges == 2 && plan.partitions[1].transferred_bytes == 8, "whole partition");
    check(plan.active_partition_count() == 1 && plan.transferred_byte_count() == 8, "plan totals");
    const auto all = transfer::ExpTMFilter(false).plan(g, parts, a);
    check(all.transferred_partition_count() == 3 && all.transferred_edge_count() == 4, "disabled = transfer all");
    throws<std::invalid_argument>([&] { (void)transfer::ExpTMFilter().plan(g, parts, ActivityTracker(5)); },
                                  "filter activity mismatch");
    const std::vector<LogicalPartition> gap = {{0, 1, 0, 2, 64}, {2, 4, 3, 4, 64}};
    throws<std::invalid_argument>([&] { (void)transfer::ExpTMFilter().plan(g, gap, a); }, "filter coverage");
}

void test_compaction() {
    const CSRGraph g = small_graph();
    const std::vector<LogicalPartition> parts = {{0, 2, 0, 3, 64}, {2, 4, 3, 4, 64}};
    ActivityTracker a(4);
    a.set_active(0);
    a.set_active(1);
    a.set_active(3);  // zero-degree active vertex
    const auto r = transfer::ExpTMCompaction().compact(g, parts, a);
    check(r.partitions.size() == 2, "both partitions have an active vertex");
    const auto &p0 = r.partitions[0];
    check(p0.active_vertices == std::vector<CSRGraph::vertex_id>({0, 1}), "active vertices");
    check(p0.neighbors == std::vector<CSRGraph::vertex_id>({1, 2, 2}), "packed neighbors");
    check(p0.neighbor_index == std::vector<CSRGraph::offset_type>({0, 2, 3}), "index with leading 0");
    check(p0.total_bytes() == 3 * 4 + 3 * 8, "payload bytes");
    const auto &p1 = r.partitions[1];
    check(p1.active_vertices == std::vector<CSRGraph::vertex_id>({3}) && p1.neighbors.empty() &&
              p1.neighbor_index == std::vector<CSRGraph::offset_type>({0, 0}),
          "zero-degree active vertex");
    check(transfer::ExpTMCompaction::expanded_neighbors(p0) == p0.neighbors, "expanded");
    auto bad = p0;
    bad.neighbor_index.back() = 7;
    throws<std::invalid_argument>([&] { (void)transfer::ExpTMCompaction::expanded_neighbors(bad); }, "bad index");
    check(transfer::ExpTMCompaction(false).compact(g, parts, a).partitions.empty(), "disabled");
    throws<std::invalid_argument>([&] { (void)transfer::ExpTMCompaction().compact(g, parts, ActivityTracker(3)); },
                                  "compaction activity mismatch");
    const std::vector<LogicalPartition> split_row = {{0, 2, 1, 3, 64}};
    throws<std::invalid_argument>([&] { (void)transfer::ExpTMCompaction().compact(g, split_row, a); },
                                  "partition not on a row boundary");
}

void test_zero_copy() {
    // vertex 0: 40 edges (160 B), vertex 1: 1 edge at byte offset 160 (unaligned)
    std::vector<CSRGraph::vertex_id> cols(41, 2);
    const CSRGraph g(3, {0, 40, 41, 41}, cols);
    const std::vector<LogicalPartition> parts = {{0, 3, 0, 41, 1024}};
    ActivityTracker a(3);
    a.set_active(0);
    a.set_active(1);
    a.set_active(2);
    const auto r = transfer::ImpTMZeroCopy().prepare(g, parts, a);
    const auto &p = r.partitions[0];
    check(p.vertex_metrics[0].memory_requests == 2 && p.vertex_metrics[0].alignment_overhead == 0, "v0 requests");
    check(p.vertex_metrics[1].memory_requests == 1 && p.vertex_metrics[1].alignment_overhead == 1, "v1 unaligned");
    check(p.vertex_metrics[2].memory_requests == 0 && p.vertex_metrics[2].alignment_overhead == 0, "v2 empty row");
    check(r.memory_request_count == 3 && r.alignment_overhead_count == 1 && r.modeled_tlp_count == 1, "totals");
    check(r.mode == transfer::ZeroCopyMode::Modeled && !r.host_memory_mapped, "prepare is metrics only");
    transfer::ZeroCopyOptions o;
    o.request_payload_bytes = 32;
    const auto r32 = transfer::ImpTMZeroCopy(o).prepare(g, parts, a);
    check(r32.partitions[0].vertex_metrics[0].memory_requests == 5, "32-byte payload");
    o.request_payload_bytes = 0;
    throws<std::invalid_argument>([&] { (void)transfer::ImpTMZeroCopy(o).prepare(g, parts, a); }, "zero payload");
    const std::vector<LogicalPartition> misaligned = {{0, 2, 0, 40, 64}, {2, 3, 40, 41, 64}};
    throws<std::invalid_argument>([&] { (void)transfer::ImpTMZeroCopy().prepare(g, misaligned, a); }, "row boundary");
}

void test_cost_model() {
    // Known answer (reference tests/unit_tests.cpp:2058-2158).
    const CSRGraph g(4, {0, 2, 3, 4, 4}, {1, 2, 2, 0});
    ActivityTracker a(4);
    a.set_active_vertices({0, 1});
    transfer::HyTMCostModelOptions o;
    o.rtt = 2.0;
    o.cpu_compaction_throughput_bytes_per_second = 14.0;
    const auto c = transfer::HyTMCostModel(o).evaluate_partition(g, LogicalPartition(0, 2, 0, 3, 1024), a);
    check(c.metrics.active_vertices == 2 && c.metrics.active_edges == 3 && c.metrics.total_edges == 3, "metrics");
    check(c.metrics.filter_transfer_bytes == 12 && close(c.filter_cost, 2.0), "filter");
    check(c.metrics.compaction_bytes == 28 && close(c.compaction_cost, 4.0), "compaction");
    check(c.metrics.zero_copy_memory_requests == 2 && c.metrics.zero_copy_alignment_overhead == 1 &&
              c.metrics.zero_copy_total_requests == 3,
          "zero-copy requests");
    check(close(c.zero_copy_rtt, 2.0) && close(c.zero_copy_cost, 2.0), "zero-copy cost");
    check(c.selected_engine == TransferEngine::ImpTMZeroCopy, "F == Z falls to zero-copy");
    // Strict selector boundaries (reference tests/unit_tests.cpp:2159-2204).
    using M = transfer::HyTMCostModel;
    check(M::select_engine(10, 7, 20, .8, .4) == TransferEngine::ExpTMCompaction, "C wins");
    check(M::select_engine(10, 8, 20, .8, .4) == TransferEngine::ExpTMFilter, "alpha strict");
    check(M::select_engine(10, 20, 10, .8, .4) == TransferEngine::ImpTMZeroCopy, "F == Z strict");
    check(M::select_engine(20, 8, 20, .8, .4) == TransferEngine::ImpTMZeroCopy, "beta strict");
    throws<std::invalid_argument>([] { (void)M::select_engine(-1, 1, 1, .8, .4); }, "negative cost");
    auto bad = o;
    bad.gamma = 1.5;
    throws<std::invalid_argument>([&] { transfer::HyTMCostModel{bad}; }, "gamma range");
    bad = o;
    bad.alpha = 0.0;
    throws<std::invalid_argument>([&] { transfer::HyTMCostModel{bad}; }, "alpha positive");
    // evaluate_metrics reproduces evaluate_partition from the same metrics
    const auto again = transfer::HyTMCostModel(o).evaluate_metrics(c.metrics);
    check(again.filter_cost == c.filter_cost && again.compaction_cost == c.compaction_cost &&
              again.zero_copy_cost == c.zero_copy_cost && again.selected_engine == c.selected_engine,
          "evaluate_metrics");
}

void test_task_combiner() {
    using E = TransferEngine;
    const E F = E::ExpTMFilter, C = E::ExpTMCompaction, Z = E::ImpTMZeroCopy;
    const scheduling::TaskCombiner tc;
    auto p = tc.combine({F, F, F, F, F, F});
    check(p.tasks.size() == 2 && p.tasks[0].partition_count() == 4 && p.tasks[1].partition_count() == 2, "k = 4");
    check(p.metrics.filter_partitions_combined == 4 && p.metrics.task_count_reduction() == 4, "filter metrics");
    p = tc.combine({F, C, F, F, Z, F, C});
    // tasks by first partition: F[0], C[1,6], F[2,3], Z[4], F[5]
    check(p.tasks.size() == 5, "mixed task count");
    check(p.tasks[1].engine == C && p.tasks[1].partition_indices == std::vector<std::size_t>({1, 6}) &&
              p.tasks[1].end_partition_index == 7,
          "one compaction task");
    check(p.tasks[2].partition_indices == std::vector<std::size_t>({2, 3}), "consecutive filters only");
    check(p.tasks[3].engine == Z && p.tasks[4].first_partition_index == 5, "order");
    for (std::size_t i = 0; i < p.tasks.size(); ++i) check(p.tasks[i].task_index == i, "task index");
    check(tc.combine({}).tasks.empty() && tc.combine({}).metrics.logical_partition_count == 0, "empty input");
    throws<std::invalid_argument>([] { scheduling::TaskCombiner(scheduling::TaskCombinerOptions{0}); }, "k = 0");
}

// -------------------------------- runtime -------------------------------
void test_runtime() {
    runtime::Config c;
    c.set("scale", "24");
    c.set("rate", "2.5");
    c.set("flag", "On");
    check(c.get_int("scale") == 24 && close(c.get_double("rate"), 2.5) && c.get_bool("flag"), "typed getters");
    check(c.get_or("missing", "x") == "x" && c.contains("scale"), "get_or");
    throws<std::out_of_range>([&] { (void)c.get("missing"); }, "missing key");
    throws<std::invalid_argument>([&] { c.set("", "v"); }, "empty key");
    c.set("flag", "maybe");
    throws<std::invalid_argument>([&] { (void)c.get_bool("flag"); }, "bad bool");
    runtime::Result r;
    r.experiment_id = "id\"1";
    r.config["k"] = "v";
    r.measurements["gteps"] = 1.5;
    const std::string j = runtime::result_to_json(r);
    check(j.find("\"experiment_id\": \"id\\\"1\"") != std::string::npos, "escaped id");
    check(j.find("\"gteps\": 1.5") != std::string::npos && j.find("\"k\": \"v\"") != std::string::npos, "fields");
}

// ---------------------------------- GPU ---------------------------------
void test_gpu() {
    using namespace algorithms;
    // reference tests/cuda_algorithm_tests.cu:23-56 graph; values from the
    // reference's pagerank_cpu (FP32) agree with the GPU within 1e-5.
    const CSRGraph g3(3, {0, 2, 3, 4}, {1, 2, 2, 0});
    PageRankOptions po;
    po.max_iterations = 200;
    const auto pr = pagerank_gpu(g3, po);
    check(pr.converged && pr.ranks.size() == 3, "pagerank_gpu converges");
    const float want[3] = {0.3877894878F, 0.2148107439F, 0.3973996341F};
    for (int i = 0; i < 3; ++i) check(std::fabs(pr.ranks[i] - want[i]) <= 1e-5F, "pagerank_gpu value");
    const auto cyc = pagerank_gpu(CSRGraph(3, {0, 1, 2, 3}, {1, 2, 0}));
    for (float r : cyc.ranks) check(std::fabs(r - 1.F / 3.F) <= 1e-5F, "cycle uniform");
    const auto dang = pagerank_gpu(CSRGraph(3, {0, 1, 2, 2}, {1, 0}));
    check(std::fabs(dang.ranks[0] + dang.ranks[1] + dang.ranks[2] - 1.F) <= 1e-5F, "mass preserved");
    PageRankOptions bad;
    bad.damping_factor = 1.0F;
    throws<std::invalid_argument>([&] { (void)pagerank_gpu(g3, bad); }, "damping 1");
    throws<std::invalid_argument>([&] { (void)pagerank_gpu(CSRGraph(0, {0}, {})); }, "empty graph");

    const CSRGraph w(4, {0, 2, 4, 5, 5}, {1, 2, 2, 3, 3}, {1.F, 4.F, 2.F, 6.F, 1.F});
    const auto s = sssp_gpu(w);
    check(s.converged && s.distances == std::vector<float>({0.F, 1.F, 3.F, 4.F}), "weighted sssp");
    const auto u = sssp_gpu(CSRGraph(4, {0, 1, 2, 2, 2}, {1, 2}));
    check(u.distances[0] == 0.F && u.distances[1] == 1.F && u.distances[2] == 2.F && std::isinf(u.distances[3]),
          "unweighted + unreachable");
    const auto x = sssp_gpu_u32(w);
    check(x.distances == std::vector<uint32_t>({0, 1, 3, 4}), "u32 distances");
    throws<std::invalid_argument>([] { (void)sssp_gpu(CSRGraph(2, {0, 1, 1}, {1}, {-1.F})); }, "negative weight");
    SSSPOptions so;
    so.source = 2;
    throws<std::invalid_argument>([&] { (void)sssp_gpu(CSRGraph(2, {0, 0, 0}, {}), so); }, "source range");

    // Reordering and hub sorting (GPU): reference tests/unit_tests.cpp:2468-2740.
    CSRGraph rw(3, {0, 2, 3, 3}, {1, 2, 2}, {5.F, 6.F, 7.F});
    rw.reorder_vertices({2, 0, 1});  // new0 = old2, new1 = old0, new2 = old1
    check(rw.row_offsets() == std::vector<CSRGraph::offset_type>({0, 0, 2, 3}), "reorder offsets");
    check(rw.column_indices() == std::vector<CSRGraph::vertex_id>({2, 0, 0}), "reorder columns");
    check(rw.edge_weights() == std::vector<float>({5.F, 6.F, 7.F}), "reorder weights");
    CSRGraph r3(3, {0, 2, 3, 4}, {1, 2, 2, 0}, {1.F, 2.F, 3.F, 4.F});
    r3.reorder_vertices({2, 0, 1});
    check(r3.row_offsets() == std::vector<CSRGraph::offset_type>({0, 1, 3, 4}), "reorder offsets 2");
    check(r3.column_indices() == std::vector<CSRGraph::vertex_id>({1, 2, 0, 0}), "reorder columns 2");
    check(r3.edge_weights() == std::vector<float>({4.F, 1.F, 2.F, 3.F}), "reorder weights 2");
    r3.validate();
    throws<std::invalid_argument>([&] { rw.reorder_vertices({0, 0, 1}); }, "duplicate order");
    throws<std::invalid_argument>([&] { rw.reorder_vertices({0, 1, 3}); }, "out-of-range order");

    using scheduling::HubSorter;
    using scheduling::HubSortOptions;
    HubSortOptions ho;
    ho.hub_fraction = 2.0 / 3.0;
    const auto sc = HubSorter(ho).sort(CSRGraph(3, {0, 2, 3, 4}, {1, 2, 2, 0}));
    check(sc.scores == std::vector<double>({0.5, 0.25, 0.5}) && sc.hub_count == 2, "hub scores");
    check(sc.vertex_order == std::vector<CSRGraph::vertex_id>({0, 2, 1}), "hub order ties by id");
    ho.hub_fraction = 0.4;
    CSRGraph h5(5, {0, 3, 4, 5, 6, 7}, {1, 2, 3, 0, 0, 0, 0});
    const auto hs = HubSorter(ho).sort(h5);
    check(hs.hub_count == 2 && hs.vertex_order == std::vector<CSRGraph::vertex_id>({0, 1, 2, 3, 4}), "hubs first");
    h5.reorder_vertices(hs.vertex_order);
    check(h5.column_indices() == std::vector<CSRGraph::vertex_id>({1, 2, 3, 0, 0, 0, 0}), "hub reorder");
    const auto el = HubSorter().sort(CSRGraph(4, {0, 0, 0, 0, 0}, {}));
    check(el.hub_count == 1 && el.vertex_order == std::vector<CSRGraph::vertex_id>({0, 1, 2, 3}), "edgeless");
    check(el.scores == std::vector<double>(4, 0.0), "edgeless scores");
    check(HubSorter().sort(CSRGraph(0, {0}, {})).empty(), "empty graph");
    // GraphLoader (GPU construction): reference tests/unit_tests.cpp:374-599.
    const std::string dir = "/tmp/hyt_dropin_" + std::to_string(::getpid());
    const std::string f1 = dir + "_unweighted.el", f2 = dir + "_weighted.el", f3 = dir + "_bad.el",
                      f4 = dir + ".csr";
    std::ofstream(f1) << "# simple directed graph\n0 1\n0 2\n1 2\n2 0\n";
    std::ofstream(f2) << "# weighted graph\n0 1 0.5\n0 2 1.25\n1 2 2.5\n";
    std::ofstream(f3) << "0 1\n0 3\n";
    const auto lg = graph::GraphLoader::load_edge_list(f1, 4, false);
    check(lg.num_edges() == 4 && lg.out_degree(0) == 2 && lg.out_degree(3) == 0 && lg.neighbor_at(3) == 0,
          "loaded unweighted graph");
    const auto lw = graph::GraphLoader::load_edge_list(f2, 3, true);
    check(lw.has_weights() && lw.weight_at(1) == 1.25F, "loaded weighted graph");
    throws<std::invalid_argument>([&] { (void)graph::GraphLoader::load_edge_list(f3, 3, false); }, "id range");
    throws<std::runtime_error>([&] { (void)graph::GraphLoader::load_edge_list(dir + "_none", 3, false); },
                               "missing file");
    graph::GraphLoader::save_csr(lw, f4);
    const auto back = graph::GraphLoader::load_csr(f4);
    check(back.row_offsets() == lw.row_offsets() && back.column_indices() == lw.column_indices() &&
              back.edge_weights() == lw.edge_weights(),
          "binary CSR round trip");
    for (const auto &f : {f1, f2, f3, f4}) std::remove(f.c_str());

    // ContributionScheduler (GPU): reference tests/unit_tests.cpp:2751-2880.
    using scheduling::ContributionPriority;
    using scheduling::ContributionScheduler;
    const auto cp = ContributionScheduler().schedule({{0U, 0.10}, {1U, 0.90}, {2U, 0.30}, {3U, 0.70}});
    check(cp.ordered_item_indices == std::vector<std::size_t>({1U, 3U, 2U, 0U}) &&
              std::fabs(cp.metrics.scheduling_overhead - 2.0) < 1e-12,
          "contribution order");
    check(ContributionScheduler().schedule({{3U, 0.5}, {1U, 0.5}, {2U, 0.9}, {0U, 0.5}}).ordered_item_indices ==
              std::vector<std::size_t>({2U, 0U, 1U, 3U}),
          "contribution ties");
    scheduling::ContributionSchedulerOptions zo;
    zo.zero_contribution_epsilon = 1e-6;
    check(ContributionScheduler(zo).schedule({{0U, 0.0}, {1U, 1e-8}, {2U, 0.25}, {3U, -1e-8}})
                  .metrics.zero_contribution_count == 3U,
          "zero contributions");
    throws<std::invalid_argument>(
        [] { (void)ContributionScheduler().schedule({{0U, std::numeric_limits<double>::infinity()}}); },
        "non-finite contribution");
    const auto pc = pagerank_contributions_gpu(CSRGraph(3, {0, 2, 3, 3}, {1, 2, 2}), {1.F, 0.F, 0.F});
    check(std::fabs(pc[0].contribution - 0.95) < 1e-5 && std::fabs(pc[1].contribution - 0.475) < 1e-5 &&
              std::fabs(pc[2].contribution - 0.475) < 1e-5,
          "pagerank contributions");
    const auto sc2 = sssp_contributions_gpu({0.F, 5.F, std::numeric_limits<float>::infinity(), 10.F},
                                            {0.F, 3.F, 7.F, 12.F});
    check(sc2[0].contribution == 0.0 && sc2[1].contribution == 2.0 && sc2[2].contribution == 1.0 &&
              sc2[3].contribution == 0.0,
          "sssp contributions");

    HubSortOptions bad_fraction;
    bad_fraction.hub_fraction = 1.5;
    throws<std::invalid_argument>([&] { HubSorter h{bad_fraction}; (void)h; }, "fraction range");
}

}  // namespace

int main(int argc, char **argv) {
    const std::string mode = argc > 1 ? argv[1] : "cpu";
    const std::vector<std::pair<const char *, std::function<void()>>> cpu = {
        {"csr", test_csr},           {"activity", test_activity}, {"partitioner", test_partitioner},
        {"filter", test_filter},     {"compaction", test_compaction}, {"zero_copy", test_zero_copy},
        {"cost_model", test_cost_model}, {"task_combiner", test_task_combiner}, {"runtime", test_runtime}};
    try {
        if (mode == "gpu") {
            int n = 0;
            if (hyt_device_count(&n) != HYT_OK || n == 0) {
                std::cout << "no CUDA device: skipped\n";
                return 77;
            }
            test_gpu();
        } else {
            for (const auto &[name, fn] : cpu) {
                fn();
                std::cout << "ok " << name << '\n';
            }
        }
    } catch (const std::exception &e) {
        std::cerr << "FAIL: " << e.what() << '\n';
        return 1;
    }
    std::cout << g_checks << " checks passed (" << mode << ")\n";
    return 0;
}
