// Multi-query engine: many SSSP and personalized-PageRank queries over many
// device-resident graphs advanced together, one superstep (one SSSP round
// and one PPR iteration of every running query) at a time.
//
// Device layout: a slot table (one slot per running query) holding each
// query's solver arguments -- the same SSArgs / PRArgs the single-query
// solvers use, pointing at the query's graph and at its own state block
// (labels, frontiers, far piles / ranks, contributions, partials).  State
// blocks come from a stream-ordered memory pool; the host admits a query
// only while the bytes of all admitted state blocks stay within the
// engine's budget.
//
// A superstep is five kernels over the whole table:
//   split  -- far-pile splits of SSSP queries whose near frontier ran dry;
//   prep   -- per-slot work units (32-vertex frontier blocks / PPR tasks)
//             and their exclusive prefix;
//   work   -- persistent grid; each warp takes units round-robin, finds the
//             slot by binary search over the prefix, and runs the same warp
//             code as the single-query kernels (expand_warp, chunk_task,
//             tile_task); long SSSP rows become hub tasks;
//   hub    -- the hub tasks of every SSSP query;
//   end    -- one CTA per slot: SSSP round end; PPR residual / dangling
//             mass summed from per-task partials in a fixed order (so a
//             query's result does not depend on the other queries in the
//             table) and the stop rule.
// hyt_batch_run captures the superstep once as the body of a conditional
// while-node, so a whole batch is one CUDA-graph launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"
#include "graph.cuh"
#include "hyt/capi.h"

namespace hyt {

struct EngineArgs;  // device-side table (batch.cu)
struct EngineHost;  // host mirrors of the table (batch.cu)

struct BatchTuning {
    uint32_t delta_mult = 0;    // SSSP bucket width = delta_mult * mean weight; 0 = one bucket
    uint32_t hub_degree = 64;   // SSSP rows at least this long become hub tasks
    uint32_t ctas_per_sm = 0;   // persistent work grid (0 = occupancy)
};

class QueryEngine {
public:
    QueryEngine(int device, cudaStream_t stream, uint64_t budget_bytes);
    ~QueryEngine();
    QueryEngine(const QueryEngine &) = delete;
    QueryEngine &operator=(const QueryEngine &) = delete;

    // Graphs are borrowed (the caller keeps them alive); index = graph id.
    void set_graphs(const std::vector<GraphImpl *> &graphs);
    void set_tuning(const BatchTuning &t) { tuning_ = t; }
    const BatchTuning &tuning() const { return tuning_; }

    // Checks a query against its graph; throws HYT_E_INVALID with the
    // single-query solvers' messages.
    void validate(const hyt_query &q) const;
    // Device bytes of a query's state block.
    uint64_t state_bytes(const hyt_query &q) const;
    uint64_t budget() const { return budget_; }
    uint64_t bytes_in_use() const { return in_use_; }

    // Admits a query into a free slot (state block allocated and
    // initialised on the stream); returns the slot, or -1 when the budget
    // or the slot capacity does not allow it now.
    int admit(const hyt_query &q, uint64_t tag);
    // Number of running (admitted, not finished) queries.
    uint32_t running() const { return running_; }
    uint32_t slots_in_use() const { return used_slots_; }

    // Runs supersteps until every admitted query is done: one CUDA-graph
    // launch with a conditional while-loop (or host-driven when
    // use_graph is false).  Returns supersteps executed.
    uint32_t run_to_completion(bool use_graph);
    // Runs exactly `n` supersteps (host-driven, for continuous batching).
    void run_supersteps(uint32_t n);
    // Enqueues one superstep as one CUDA-graph launch (no conditional).
    void step();

    // Slots whose query finished (synchronises the stream).  Each entry:
    // slot, tag.
    std::vector<std::pair<int, uint64_t>> finished();
    // Copies a finished query's result to its `out` pointer (stream-ordered)
    // and fills `res`; frees the slot and its state block.
    void retire(int slot, hyt_query_result *res);

    // Drops every admitted query (after a failed run): frees the state
    // blocks and clears the table.
    void reset();

    cudaStream_t stream() const { return stream_; }
    uint64_t launches() const { return launches_; }

private:
    struct SlotHost {
        bool used = false, running = false;
        hyt_query q{};
        uint64_t tag = 0, bytes = 0, hub = 0;
        void *mem = nullptr;
    };
    void grow(uint32_t cap);
    void ensure_hub_capacity();
    void build_graph_exec();
    void build_step_exec();
    void add_superstep_nodes(cudaGraph_t body, int grid);
    void upload_args(bool use_cond);
    void launch_superstep_kernels(cudaStream_t s);
    int work_grid() const;
    int ppr_grid() const;

    int device_;
    cudaStream_t stream_;
    uint64_t budget_, in_use_ = 0;
    std::vector<GraphImpl *> graphs_;
    BatchTuning tuning_;
    std::vector<SlotHost> slots_;
    uint32_t cap_ = 0, hi_ = 0, used_slots_ = 0, running_ = 0, max_supersteps_ = 1;
    uint64_t hub_need_ = 0, launches_ = 0;
    cudaMemPool_t pool_ = nullptr;
    std::unique_ptr<EngineHost> host_;  // host mirrors and device copies of the slot table

    DeviceArray<uint32_t> unit_base_;   // [cap + 1]
    DeviceArray<uint4> hubs_;
    DeviceArray<uint32_t> counters_;    // hub tasks, running, supersteps, overflow
    DeviceArray<EngineArgs> d_args_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphConditionalHandle cond_{};
    int exec_grid_ = 0;
    cudaGraph_t step_graph_ = nullptr;
    cudaGraphExec_t step_exec_ = nullptr;
    int step_grid_ = 0;
    bool args_dirty_ = true;

public:
    uint64_t frontier_total = 0;  // SSSP frontier vertices of retired queries
};

}  // namespace hyt

struct hyt_batch {
    std::vector<hyt::GraphImpl *> graphs;
    hyt::QueryEngine *engine = nullptr;
    hyt::BatchTuning tuning;
    cudaStream_t stream = nullptr;
    int device = 0;
    uint32_t flags = 0;
};
