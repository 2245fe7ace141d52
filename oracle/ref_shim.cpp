// ref_shim.cpp -- extern "C" wrappers around the REFERENCE's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
// with the reference's sources (read in place from the reference checkout,
// never copied) into oracle/_ref/libhytref.so.  Tests use it to pin the
// oracle restatement (oracle.c) and the product's host logic; bench.py
// --impl reference times ref_pagerank_cpu / ref_sssp_cpu as the CPU arm.
//
// Compiled against the reference's headers only (-I <reference>/include).
#include "algorithms/pagerank.hpp"
#include "algorithms/sssp.hpp"
#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"
#include "graph/graph_loader.hpp"
#include "scheduling/contribution_scheduler.hpp"
#include "scheduling/hub_sort.hpp"
#include "scheduling/task_combiner.hpp"
#include "transfer/compaction_engine.hpp"
#include "transfer/filter_engine.hpp"
#include "transfer/hytm_cost_model.hpp"
#include "transfer/zero_copy_engine.hpp"

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {
thread_local std::string g_err;

int fail_code(const std::exception &e, int code) {
    g_err = e.what();
    return code;
}

hytgraph::graph::CSRGraph make_graph(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols,
                                     const float *w) {
    std::vector<uint64_t> o(off, off + V + 1);
    std::vector<uint32_t> c(cols, cols + E);
    std::vector<float> wt;
    if (w) wt.assign(w, w + E);
    return hytgraph::graph::CSRGraph(V, std::move(o), std::move(c), std::move(wt));
}

#define REF_GUARD(...)                                      \
    try {                                                   \
        __VA_ARGS__;                                           \
        return 0;                                           \
    } catch (const std::invalid_argument &e) {              \
        return fail_code(e, 1);                             \
    } catch (const std::out_of_range &e) {                  \
        return fail_code(e, 3);                             \
    } catch (const std::exception &e) {                     \
        return fail_code(e, 2);                             \
    }
}  // namespace

#pragma GCC visibility push(default)
extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

int ref_pagerank_cpu(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, float damping, float tol,
                     uint64_t max_iter, float *ranks, uint64_t *iterations, float *residual, int *converged) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::algorithms::PageRankOptions o;
        o.damping_factor = damping;
        o.tolerance = tol;
        o.max_iterations = max_iter;
        const auto r = hytgraph::algorithms::pagerank_cpu(g, o);
        std::memcpy(ranks, r.ranks.data(), r.ranks.size() * sizeof(float));
        *iterations = r.iterations;
        *residual = r.residual;
        *converged = r.converged ? 1 : 0;
    })
}

int ref_sssp_cpu(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *w, uint32_t source,
                 uint64_t max_iter, float *dist, uint64_t *iterations, int *converged) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, w);
        hytgraph::algorithms::SSSPOptions o;
        o.source = source;
        o.max_iterations = max_iter;
        const auto r = hytgraph::algorithms::sssp_cpu(g, o);
        std::memcpy(dist, r.distances.data(), r.distances.size() * sizeof(float));
        *iterations = r.iterations;
        *converged = r.converged ? 1 : 0;
    })
}

// Per-partition HyTM costs.  parts: n x {vbegin, vend} (edge bounds taken
// from the CSR); opts: alpha, beta, gamma, rtt, cpu_throughput (doubles) and
// m, mr (u64).  Outputs per partition: metrics[11] (u64: vbegin, vend,
// active_vertices, active_edges, total_edges, filter_bytes, compaction_bytes,
// zc_requests, zc_alignment, zc_total, partition_index), costs[4] (filter,
// compaction, zero_copy, zc_rtt) and engine (0 F, 1 C, 2 Z).
int ref_hytm_evaluate(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const unsigned char *active,
                      uint64_t nparts, const uint32_t *parts, const double *dopts, const uint64_t *uopts,
                      uint64_t *metrics, double *costs, int *engines) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::graph::ActivityTracker act(V);
        for (uint64_t v = 0; v < V; ++v)
            if (active[v]) act.set_active(static_cast<uint32_t>(v));
        std::vector<hytgraph::graph::LogicalPartition> ps;
        for (uint64_t i = 0; i < nparts; ++i)
            ps.emplace_back(parts[2 * i], parts[2 * i + 1], off[parts[2 * i]], off[parts[2 * i + 1]], 1u << 20);
        hytgraph::transfer::HyTMCostModelOptions o;
        o.alpha = dopts[0];
        o.beta = dopts[1];
        o.gamma = dopts[2];
        o.rtt = dopts[3];
        o.cpu_compaction_throughput_bytes_per_second = dopts[4];
        o.request_payload_bytes = uopts[0];
        o.max_requests_per_tlp = uopts[1];
        const hytgraph::transfer::HyTMCostModel model(o);
        const auto r = model.evaluate_partitions(g, ps, act);
        for (uint64_t i = 0; i < nparts; ++i) {
            const auto &m = r[i].metrics;
            uint64_t *mo = metrics + 11 * i;
            mo[0] = m.vertex_begin; mo[1] = m.vertex_end; mo[2] = m.active_vertices; mo[3] = m.active_edges;
            mo[4] = m.total_edges; mo[5] = m.filter_transfer_bytes; mo[6] = m.compaction_bytes;
            mo[7] = m.zero_copy_memory_requests; mo[8] = m.zero_copy_alignment_overhead;
            mo[9] = m.zero_copy_total_requests; mo[10] = m.partition_index;
            costs[4 * i + 0] = r[i].filter_cost;
            costs[4 * i + 1] = r[i].compaction_cost;
            costs[4 * i + 2] = r[i].zero_copy_cost;
            costs[4 * i + 3] = r[i].zero_copy_rtt;
            engines[i] = static_cast<int>(r[i].selected_engine);
        }
    })
}

int ref_select_engine(double f, double c, double z, double alpha, double beta, int *engine) {
    REF_GUARD({ *engine = static_cast<int>(hytgraph::transfer::HyTMCostModel::select_engine(f, c, z, alpha, beta)); })
}

// Task combining: engines[n] -> per partition its task index; per task its
// engine and first partition.  Returns the task count in *ntasks.
int ref_task_combine(const int *engines, uint64_t n, uint64_t k, uint64_t *task_of_partition, int *task_engine,
                     uint64_t *task_first, uint64_t *ntasks, uint64_t *metrics) {
    REF_GUARD({
        std::vector<hytgraph::transfer::TransferEngine> es;
        for (uint64_t i = 0; i < n; ++i) es.push_back(static_cast<hytgraph::transfer::TransferEngine>(engines[i]));
        hytgraph::scheduling::TaskCombinerOptions o;
        o.filter_combine_k = k;
        const auto plan = hytgraph::scheduling::TaskCombiner(o).combine(es);
        *ntasks = plan.tasks.size();
        for (const auto &t : plan.tasks) {
            task_engine[t.task_index] = static_cast<int>(t.engine);
            task_first[t.task_index] = t.first_partition_index;
            for (const auto p : t.partition_indices) task_of_partition[p] = t.task_index;
        }
        metrics[0] = plan.metrics.logical_partition_count;
        metrics[1] = plan.metrics.executable_task_count;
        metrics[2] = plan.metrics.filter_partitions_combined;
        metrics[3] = plan.metrics.compaction_partitions_combined;
        metrics[4] = plan.metrics.zero_copy_partitions_combined;
    })
}

// GraphLoader::load_edge_list: loads into a holder, *E_out = edge count;
// ref_loaded_copy then copies the arrays out (w may be NULL).
static hytgraph::graph::CSRGraph g_loaded;
int ref_load_edge_list(const char *path, uint64_t V, int weighted, uint64_t *E_out) {
    REF_GUARD({
        g_loaded = hytgraph::graph::GraphLoader::load_edge_list(path, V, weighted != 0);
        *E_out = g_loaded.num_edges();
    })
}
void ref_loaded_copy(uint64_t *off, uint32_t *cols, float *w) {
    const auto &o = g_loaded.row_offsets();
    const auto &c = g_loaded.column_indices();
    const auto &x = g_loaded.edge_weights();
    for (size_t i = 0; i < o.size(); ++i) off[i] = o[i];
    for (size_t i = 0; i < c.size(); ++i) cols[i] = c[i];
    if (w)
        for (size_t i = 0; i < x.size(); ++i) w[i] = x[i];
}

// pagerank_contributions: out[V] (vertex order as returned).
int ref_pagerank_contributions(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *cur,
                               float damping, double *out) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::algorithms::PageRankOptions o;
        o.damping_factor = damping;
        const auto r = hytgraph::algorithms::pagerank_contributions(g, std::vector<float>(cur, cur + V), o);
        for (const auto &c : r) out[c.vertex] = c.contribution;
    })
}

int ref_sssp_contributions(uint64_t n, const float *cur, const float *cand, float tol, double *out) {
    REF_GUARD({
        const auto r = hytgraph::algorithms::sssp_contributions(std::vector<float>(cur, cur + n),
                                                                std::vector<float>(cand, cand + n), tol);
        for (const auto &c : r) out[c.vertex] = c.contribution;
    })
}

// ContributionScheduler::schedule: ordered[n]; metrics[7] as in the oracle.
int ref_contribution_schedule(uint64_t n, const uint64_t *item, const double *c, int det, double eps, uint64_t *ordered,
                              uint64_t *metrics) {
    REF_GUARD({
        hytgraph::scheduling::ContributionSchedulerOptions o;
        o.deterministic_tie_break = det != 0;
        o.zero_contribution_epsilon = eps;
        std::vector<hytgraph::scheduling::ContributionPriority> p(n);
        for (uint64_t i = 0; i < n; ++i) p[i] = {static_cast<std::size_t>(item[i]), c[i]};
        const auto plan = hytgraph::scheduling::ContributionScheduler(o).schedule(p);
        for (uint64_t i = 0; i < n; ++i) ordered[i] = plan.ordered_item_indices[i];
        const auto &m = plan.metrics;
        metrics[0] = m.input_item_count;
        metrics[1] = m.scheduled_item_count;
        metrics[2] = m.reordered_item_count;
        metrics[3] = m.zero_contribution_count;
        std::memcpy(&metrics[4], &m.scheduling_overhead, 8);
        metrics[5] = m.stale_work_count;
        metrics[6] = m.redundant_work_count;
    })
}

// HubSorter::sort: vertex_order[V], scores[V], hub_count.
int ref_hub_sort(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, double fraction,
                 uint32_t *order, double *scores, uint64_t *hub_count) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::scheduling::HubSortOptions o;
        o.hub_fraction = fraction;
        const auto r = hytgraph::scheduling::HubSorter(o).sort(g);
        for (uint64_t i = 0; i < r.vertex_order.size(); ++i) order[i] = r.vertex_order[i];
        for (uint64_t i = 0; i < r.scores.size(); ++i) scores[i] = r.scores[i];
        *hub_count = r.hub_count;
    })
}

// CSRGraph::reorder_vertices: outputs the reordered arrays (w may be NULL).
int ref_reorder(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *w,
                const uint32_t *order, uint64_t *off_out, uint32_t *cols_out, float *w_out) {
    REF_GUARD({
        auto g = make_graph(V, E, off, cols, w);
        g.reorder_vertices(std::vector<uint32_t>(order, order + V));
        for (uint64_t v = 0; v <= V; ++v) off_out[v] = g.row_offsets()[v];
        for (uint64_t e = 0; e < E; ++e) cols_out[e] = g.column_indices()[e];
        if (w && w_out)
            for (uint64_t e = 0; e < E; ++e) w_out[e] = g.edge_weights()[e];
    })
}

// Logical partitioning by target bytes: writes up to cap {vbegin, vend}.
int ref_partition(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, uint64_t target_bytes,
                  uint64_t cap, uint32_t *parts, uint64_t *nparts) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        const auto ps = hytgraph::graph::LogicalPartitioner(target_bytes).partition(g);
        *nparts = ps.size();
        for (uint64_t i = 0; i < ps.size() && i < cap; ++i) {
            parts[2 * i] = ps[i].vertex_begin();
            parts[2 * i + 1] = ps[i].vertex_end();
        }
    })
}

// Filter plan / compaction payload / zero-copy metrics over given partitions.
// filter_out per partition: {active, transferred, active_edges, total_edges,
// transferred_edges, transferred_bytes}.
int ref_filter_plan(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const unsigned char *active,
                    uint64_t nparts, const uint32_t *parts, int enabled, uint64_t *filter_out) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::graph::ActivityTracker act(V);
        for (uint64_t v = 0; v < V; ++v)
            if (active[v]) act.set_active(static_cast<uint32_t>(v));
        std::vector<hytgraph::graph::LogicalPartition> ps;
        for (uint64_t i = 0; i < nparts; ++i)
            ps.emplace_back(parts[2 * i], parts[2 * i + 1], off[parts[2 * i]], off[parts[2 * i + 1]], 1u << 20);
        const auto plan = hytgraph::transfer::ExpTMFilter(enabled != 0).plan(g, ps, act);
        for (uint64_t i = 0; i < nparts; ++i) {
            const auto &d = plan.partitions[i];
            uint64_t *o = filter_out + 6 * i;
            o[0] = d.active; o[1] = d.transferred; o[2] = d.active_edges; o[3] = d.total_edges;
            o[4] = d.transferred_edges; o[5] = d.transferred_bytes;
        }
    })
}

// Compaction: concatenated payloads of all compacted partitions.  Writes
// per compacted partition its index (cpart), and the flattened
// active_vertices / neighbors / neighbor_index streams with their lengths.
int ref_compact(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const unsigned char *active,
                uint64_t nparts, const uint32_t *parts, uint64_t *ncompacted, uint64_t *cpart, uint32_t *av,
                uint64_t *nav, uint32_t *nb, uint64_t *nnb, uint64_t *idx, uint64_t *nidx) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::graph::ActivityTracker act(V);
        for (uint64_t v = 0; v < V; ++v)
            if (active[v]) act.set_active(static_cast<uint32_t>(v));
        std::vector<hytgraph::graph::LogicalPartition> ps;
        for (uint64_t i = 0; i < nparts; ++i)
            ps.emplace_back(parts[2 * i], parts[2 * i + 1], off[parts[2 * i]], off[parts[2 * i + 1]], 1u << 20);
        const auto r = hytgraph::transfer::ExpTMCompaction(true).compact(g, ps, act);
        *ncompacted = r.partitions.size();
        uint64_t a = 0, b = 0, c = 0;
        for (uint64_t i = 0; i < r.partitions.size(); ++i) {
            const auto &p = r.partitions[i];
            cpart[i] = p.partition_index;
            for (auto x : p.active_vertices) av[a++] = x;
            for (auto x : p.neighbors) nb[b++] = x;
            for (auto x : p.neighbor_index) idx[c++] = x;
        }
        *nav = a; *nnb = b; *nidx = c;
    })
}

// Zero-copy metrics: per partition {active_vertices, active_edges, requests,
// alignment}; totals {active_partitions, requests, alignment, tlps}.
int ref_zero_copy(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const unsigned char *active,
                  uint64_t nparts, const uint32_t *parts, uint64_t payload, uint64_t mr, uint64_t *per_part,
                  uint64_t *totals) {
    REF_GUARD({
        const auto g = make_graph(V, E, off, cols, nullptr);
        hytgraph::graph::ActivityTracker act(V);
        for (uint64_t v = 0; v < V; ++v)
            if (active[v]) act.set_active(static_cast<uint32_t>(v));
        std::vector<hytgraph::graph::LogicalPartition> ps;
        for (uint64_t i = 0; i < nparts; ++i)
            ps.emplace_back(parts[2 * i], parts[2 * i + 1], off[parts[2 * i]], off[parts[2 * i + 1]], 1u << 20);
        hytgraph::transfer::ZeroCopyOptions o;
        o.request_payload_bytes = payload;
        o.max_requests_per_tlp = mr;
        const auto r = hytgraph::transfer::ImpTMZeroCopy(o).prepare(g, ps, act);
        for (uint64_t i = 0; i < nparts; ++i) {
            const auto &p = r.partitions[i];
            per_part[4 * i + 0] = p.active_vertices.size();
            per_part[4 * i + 1] = p.active_edge_count;
            per_part[4 * i + 2] = p.memory_request_count;
            per_part[4 * i + 3] = p.alignment_overhead_count;
        }
        totals[0] = r.active_partition_count;
        totals[1] = r.memory_request_count;
        totals[2] = r.alignment_overhead_count;
        totals[3] = r.modeled_tlp_count;
    })
}

}  // extern "C"
#pragma GCC visibility pop
