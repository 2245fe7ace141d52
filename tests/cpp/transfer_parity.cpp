// Randomized parity of the host-side transfer/scheduling classes against
// the reference's own compiled classes (oracle/_ref/libhytref.so, loaded
// with dlopen; its C++ symbols are hidden, so each side runs its own code).
//
//   transfer_parity <path to libhytref.so> [cases]
//
// Compares, on random R-MAT-like graphs, activity sets and partitions:
// LogicalPartitioner::partition, ExpTMFilter::plan, ExpTMCompaction::compact,
// ImpTMZeroCopy::prepare, HyTMCostModel::evaluate_partitions (metrics, costs
// bit for bit, engine) and TaskCombiner::combine.
#include "graph/activity_tracker.hpp"
#include "graph/csr_graph.hpp"
#include "graph/partition.hpp"
#include "scheduling/task_combiner.hpp"
#include "transfer/compaction_engine.hpp"
#include "transfer/filter_engine.hpp"
#include "transfer/hytm_cost_model.hpp"
#include "transfer/zero_copy_engine.hpp"

#include <dlfcn.h>

#include <cstdint>
#include <cstring>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

using namespace hytgraph;

namespace {

using u64 = uint64_t;
using u32 = uint32_t;
using u8 = unsigned char;

struct Ref {
    void *h = nullptr;
    int (*partition)(u64, u64, const u64 *, const u32 *, u64, u64, u32 *, u64 *);
    int (*filter)(u64, u64, const u64 *, const u32 *, const u8 *, u64, const u32 *, int, u64 *);
    int (*compact)(u64, u64, const u64 *, const u32 *, const u8 *, u64, const u32 *, u64 *, u64 *, u32 *, u64 *,
                   u32 *, u64 *, u64 *, u64 *);
    int (*zero_copy)(u64, u64, const u64 *, const u32 *, const u8 *, u64, const u32 *, u64, u64, u64 *, u64 *);
    int (*hytm)(u64, u64, const u64 *, const u32 *, const u8 *, u64, const u32 *, const double *, const u64 *, u64 *,
                double *, int *);
    int (*combine)(const int *, u64, u64, u64 *, int *, u64 *, u64 *, u64 *);

    explicit Ref(const char *path) {
        h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!h) throw std::runtime_error(std::string("dlopen: ") + dlerror());
        load(partition, "ref_partition");
        load(filter, "ref_filter_plan");
        load(compact, "ref_compact");
        load(zero_copy, "ref_zero_copy");
        load(hytm, "ref_hytm_evaluate");
        load(combine, "ref_task_combine");
    }
    template <class F>
    void load(F &f, const char *name) {
        f = reinterpret_cast<F>(dlsym(h, name));
        if (!f) throw std::runtime_error(std::string("missing ") + name);
    }
};

int g_checks = 0;
void check(bool ok, const std::string &what) {
    ++g_checks;
    if (!ok) throw std::runtime_error("mismatch: " + what);
}

graph::CSRGraph random_graph(std::mt19937_64 &rng, u32 V, u32 avg_deg) {
    std::vector<u64> off(V + 1, 0);
    std::vector<u32> cols;
    std::geometric_distribution<int> deg(1.0 / (1.0 + avg_deg));
    std::uniform_int_distribution<u32> dst(0, V - 1);
    for (u32 v = 0; v < V; ++v) {
        int d = deg(rng);
        if (rng() % 50 == 0) d *= 40;  // a few heavy rows
        for (int k = 0; k < d; ++k) cols.push_back(dst(rng));
        off[v + 1] = cols.size();
    }
    return graph::CSRGraph(V, std::move(off), std::move(cols));
}

void one_case(const Ref &ref, std::mt19937_64 &rng) {
    const u32 V = 1 + static_cast<u32>(rng() % 3000);
    const auto g = random_graph(rng, V, 1 + static_cast<u32>(rng() % 20));
    const u64 E = g.num_edges();
    const u64 *off = g.row_offsets().data();
    const u32 *cols = E ? g.column_indices().data() : nullptr;
    static const u32 dummy = 0;
    if (!cols) cols = &dummy;

    // ---- partitioning
    const u64 target = 4 * (1 + rng() % 2000);
    const auto parts = graph::LogicalPartitioner(target).partition(g);
    std::vector<u32> rp(2 * (V + 2));
    u64 nrp = 0;
    check(ref.partition(V, E, off, cols, target, V + 2, rp.data(), &nrp) == 0, "ref_partition rc");
    check(nrp == parts.size(), "partition count");
    std::vector<u32> pb;
    for (std::size_t i = 0; i < parts.size(); ++i) {
        check(parts[i].vertex_begin() == rp[2 * i] && parts[i].vertex_end() == rp[2 * i + 1], "partition bounds");
        pb.push_back(parts[i].vertex_begin());
        pb.push_back(parts[i].vertex_end());
    }

    // ---- activity
    graph::ActivityTracker act(V);
    std::vector<u8> flags(V, 0);
    const double frac = std::vector<double>{0.0, 0.001, 0.05, 0.3, 1.0}[rng() % 5];
    for (u32 v = 0; v < V; ++v)
        if (std::uniform_real_distribution<double>(0, 1)(rng) < frac) {
            act.set_active(v);
            flags[v] = 1;
        }

    // ---- filter
    for (int enabled = 0; enabled < 2; ++enabled) {
        const auto plan = transfer::ExpTMFilter(enabled != 0).plan(g, parts, act);
        std::vector<u64> rf(6 * parts.size());
        check(ref.filter(V, E, off, cols, flags.data(), parts.size(), pb.data(), enabled, rf.data()) == 0, "filter rc");
        for (std::size_t i = 0; i < parts.size(); ++i) {
            const auto &d = plan.partitions[i];
            const u64 *o = &rf[6 * i];
            check(d.active == (o[0] != 0) && d.transferred == (o[1] != 0) && d.active_edges == o[2] &&
                      d.total_edges == o[3] && d.transferred_edges == o[4] && d.transferred_bytes == o[5],
                  "filter decision");
        }
    }

    // ---- compaction
    const auto comp = transfer::ExpTMCompaction().compact(g, parts, act);
    std::vector<u64> cpart(parts.size()), idx(V + parts.size() + 1);
    std::vector<u32> av(V + 1), nb(E + 1);
    u64 nc = 0, nav = 0, nnb = 0, nidx = 0;
    check(ref.compact(V, E, off, cols, flags.data(), parts.size(), pb.data(), &nc, cpart.data(), av.data(), &nav,
                      nb.data(), &nnb, idx.data(), &nidx) == 0,
          "compact rc");
    check(nc == comp.partitions.size(), "compacted partition count");
    u64 a = 0, b = 0, c = 0;
    for (std::size_t i = 0; i < comp.partitions.size(); ++i) {
        const auto &p = comp.partitions[i];
        check(p.partition_index == cpart[i], "compacted index");
        for (auto x : p.active_vertices) check(x == av[a++], "active vertex");
        for (auto x : p.neighbors) check(x == nb[b++], "neighbor");
        for (auto x : p.neighbor_index) check(x == idx[c++], "neighbor index");
    }
    check(a == nav && b == nnb && c == nidx, "payload lengths");

    // ---- zero-copy
    const u64 payload = std::vector<u64>{32, 64, 96, 128}[rng() % 4];
    transfer::ZeroCopyOptions zo;
    zo.request_payload_bytes = payload;
    const auto zc = transfer::ImpTMZeroCopy(zo).prepare(g, parts, act);
    std::vector<u64> zp(4 * parts.size()), zt(4);
    check(ref.zero_copy(V, E, off, cols, flags.data(), parts.size(), pb.data(), payload, 256, zp.data(), zt.data()) ==
              0,
          "zero-copy rc");
    for (std::size_t i = 0; i < parts.size(); ++i) {
        const auto &p = zc.partitions[i];
        check(p.active_vertices.size() == zp[4 * i] && p.active_edge_count == zp[4 * i + 1] &&
                  p.memory_request_count == zp[4 * i + 2] && p.alignment_overhead_count == zp[4 * i + 3],
              "zero-copy partition");
    }
    check(zc.active_partition_count == zt[0] && zc.memory_request_count == zt[1] &&
              zc.alignment_overhead_count == zt[2] && zc.modeled_tlp_count == zt[3],
          "zero-copy totals");

    // ---- cost model
    transfer::HyTMCostModelOptions o;
    const double rtts[] = {1.0, 2.0, 3.2e-6};
    const double tputs[] = {1.0, 14.0, 2.4e10};
    o.rtt = rtts[rng() % 3];
    o.cpu_compaction_throughput_bytes_per_second = tputs[rng() % 3];
    const auto costs = transfer::HyTMCostModel(o).evaluate_partitions(g, parts, act);
    const double dopts[5] = {o.alpha, o.beta, o.gamma, o.rtt, o.cpu_compaction_throughput_bytes_per_second};
    const u64 uopts[2] = {o.request_payload_bytes, o.max_requests_per_tlp};
    std::vector<u64> m(11 * parts.size());
    std::vector<double> cc(4 * parts.size());
    std::vector<int> eng(parts.size());
    check(ref.hytm(V, E, off, cols, flags.data(), parts.size(), pb.data(), dopts, uopts, m.data(), cc.data(),
                   eng.data()) == 0,
          "hytm rc");
    std::vector<int> engines;
    for (std::size_t i = 0; i < parts.size(); ++i) {
        const auto &x = costs[i];
        const u64 *mm = &m[11 * i];
        check(x.metrics.active_vertices == mm[2] && x.metrics.active_edges == mm[3] && x.metrics.total_edges == mm[4] &&
                  x.metrics.filter_transfer_bytes == mm[5] && x.metrics.compaction_bytes == mm[6] &&
                  x.metrics.zero_copy_memory_requests == mm[7] && x.metrics.zero_copy_alignment_overhead == mm[8] &&
                  x.metrics.zero_copy_total_requests == mm[9] && x.metrics.partition_index == mm[10],
              "cost metrics");
        check(std::memcmp(&x.filter_cost, &cc[4 * i + 0], 8) == 0 && std::memcmp(&x.compaction_cost, &cc[4 * i + 1], 8) == 0 &&
                  std::memcmp(&x.zero_copy_cost, &cc[4 * i + 2], 8) == 0 &&
                  std::memcmp(&x.zero_copy_rtt, &cc[4 * i + 3], 8) == 0,
              "costs bit for bit");
        check(static_cast<int>(x.selected_engine) == eng[i], "selected engine");
        engines.push_back(eng[i]);
    }

    // ---- task combining (on the selected engines and on random ones)
    for (int round = 0; round < 2; ++round) {
        if (round == 1)
            for (auto &e : engines) e = static_cast<int>(rng() % 3);
        const u64 k = 1 + rng() % 6;
        std::vector<transfer::TransferEngine> es;
        for (int e : engines) es.push_back(static_cast<transfer::TransferEngine>(e));
        const auto plan = scheduling::TaskCombiner(scheduling::TaskCombinerOptions{k}).combine(es);
        std::vector<u64> top(es.size() + 1), tfirst(es.size() + 2), met(5);
        std::vector<int> teng(es.size() + 2);
        u64 nt = 0;
        check(ref.combine(engines.data(), es.size(), k, top.data(), teng.data(), tfirst.data(), &nt, met.data()) == 0,
              "combine rc");
        check(nt == plan.tasks.size(), "task count");
        for (const auto &t : plan.tasks) {
            check(static_cast<int>(t.engine) == teng[t.task_index] && t.first_partition_index == tfirst[t.task_index],
                  "task");
            for (auto p : t.partition_indices) check(top[p] == t.task_index, "membership");
        }
        check(plan.metrics.logical_partition_count == met[0] && plan.metrics.executable_task_count == met[1] &&
                  plan.metrics.filter_partitions_combined == met[2] &&
                  plan.metrics.compaction_partitions_combined == met[3] &&
                  plan.metrics.zero_copy_partitions_combined == met[4],
              "combine metrics");
    }
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::cerr << "usage: transfer_parity <libhytref.so> [cases]\n";
        return 2;
    }
    const int cases = argc > 2 ? std::atoi(argv[2]) : 200;
    try {
        const Ref ref(argv[1]);
        std::mt19937_64 rng(20241203);
        for (int i = 0; i < cases; ++i) one_case(ref, rng);
    } catch (const std::exception &e) {
        std::cerr << "FAIL: " << e.what() << '\n';
        return 1;
    }
    std::cout << g_checks << " parity checks passed over " << cases << " random cases\n";
    return 0;
}
