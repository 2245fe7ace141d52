// Continuous-batching query server (hyt_server_*).
//
// One worker thread drives a QueryEngine (batch.cuh) on its own stream:
//   1. take every newly submitted query (FIFO order);
//   2. admit waiting queries, oldest first, while the per-query state
//      budget, the running cap and the slot table allow (a query that does
//      not fit blocks the ones behind it: no reordering, no starvation; a
//      query that cannot fit even an idle engine completes with HYT_E_OOM);
//   3. advance every running query by one superstep (one CUDA-graph
//      launch: split, prep, work, hub, end);
//   4. retire finished queries: copy each result to the query's `out`
//      buffer, then queue its completion with its latency.
// Queries that arrive while others run join at the next superstep, and
// their work shares the superstep's kernels with everything else running.
// With nothing running the worker sleeps on a condition variable.
//
// Queries on large graphs (at least pack_min_edges edges) do not enter the
// engine: one solve there already fills the GPU, so what pays is sharing
// the graph passes between queries.  They wait in packs keyed by (graph,
// kind, restart, tolerance, iteration cap); each worker pass runs the pack
// whose oldest query is oldest, up to 8 queries at once, as one
// hyt_sssp_multi / hyt_ppr_multi solve (each query's result is what that
// solver gives it alone: SSSP labels equal hyt_sssp's), then one engine
// superstep for the small-graph queries.  A pack's state is the graph's own
// workspace, outside the per-query state budget.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <map>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "host_checks.hpp"
#include "graph.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct ServerImpl {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<GraphImpl *> graphs;
    std::unique_ptr<QueryEngine> engine;
    uint32_t max_running = 0;

    struct Pending {
        hyt_query q;
        uint64_t ticket;
        Clock::time_point submitted;
    };
    struct Running {
        Clock::time_point submitted, admitted;
    };
    // Queries of one pack share graph, kind and solver parameters.
    struct PackKey {
        uint32_t graph, kind, max_iter;
        float restart, tolerance;
        bool operator<(const PackKey &o) const {
            return std::tie(graph, kind, max_iter, restart, tolerance) <
                   std::tie(o.graph, o.kind, o.max_iter, o.restart, o.tolerance);
        }
    };
    uint64_t pack_min_edges = uint64_t(1) << 22;
    DeviceArray<uint32_t> pack_buf;  // [8][largest packed graph's V]
    uint64_t packs_run = 0;

    bool packable(const hyt_query &q) const { return graphs[q.graph]->E >= pack_min_edges; }
    static PackKey pack_key(const hyt_query &q);
    // Solves up to 8 queries of one key together; appends their completions.
    void run_pack(std::vector<Pending> &pack, std::vector<hyt_completion> &out);

    std::mutex mu;  // submissions, completions, stats
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> inbox;
    std::deque<hyt_completion> done;
    uint64_t next_ticket = 1;
    bool stop = false;
    int failure = HYT_OK;
    std::string failure_msg;
    hyt_server_stats st{};

    std::thread worker;

    void loop();
    void fail_all(const std::vector<uint64_t> &tickets, int code, const char *msg);
};

ServerImpl::PackKey ServerImpl::pack_key(const hyt_query &q) {
    PackKey k{q.graph, q.kind, q.max_iterations, 0.0f, 0.0f};
    if (q.kind == HYT_QUERY_PPR) {
        k.restart = q.restart > 0.0f ? q.restart : 0.15f;
        k.tolerance = q.tolerance > 0.0f ? q.tolerance : 1e-6f;
        if (!k.max_iter) k.max_iter = 100;
    }
    return k;
}

void ServerImpl::run_pack(std::vector<Pending> &pack, std::vector<hyt_completion> &out) {
    const PackKey key = pack_key(pack.front().q);
    GraphImpl &g = *graphs[key.graph];
    const uint32_t k = static_cast<uint32_t>(pack.size());
    const uint64_t V = g.V;
    if (pack_buf.count < 8 * V) pack_buf.allocate(8 * V);
    std::vector<uint32_t> src(k);
    for (uint32_t i = 0; i < k; ++i) src[i] = pack[i].q.source;
    hyt_run_stats st[8] = {};
    if (key.kind == HYT_QUERY_SSSP) {
        sssp_multi(g, src.data(), k, key.max_iter, 0, stream, pack_buf.get(), &st[0]);
        for (uint32_t i = 1; i < k; ++i) st[i] = st[0];
    } else {
        ppr_multi(g, src.data(), k, key.restart, key.tolerance, key.max_iter, reinterpret_cast<float *>(pack_buf.get()),
                  st);
        HYT_CUDA(cudaStreamSynchronize(g.stream));
    }
    for (uint32_t i = 0; i < k; ++i)
        if (pack[i].q.out)
            HYT_CUDA(cudaMemcpyAsync(pack[i].q.out, pack_buf.get() + i * V, V * sizeof(uint32_t), cudaMemcpyDefault,
                                     stream));
    HYT_CUDA(cudaStreamSynchronize(stream));
    const auto now = Clock::now();
    for (uint32_t i = 0; i < k; ++i) {
        hyt_completion c{};
        c.ticket = pack[i].ticket;
        c.status = HYT_OK;
        c.result.iterations = st[i].iterations;
        c.result.converged = st[i].converged;
        c.result.residual = st[i].residual;
        c.result.edges_processed = key.kind == HYT_QUERY_SSSP ? st[0].edges_processed / k : st[i].edges_processed;
        c.queue_ms = 0.0;
        c.latency_ms = ms_between(pack[i].submitted, now);
        out.push_back(c);
    }
    ++packs_run;
}

void ServerImpl::loop() {
    cudaSetDevice(device);
    std::deque<Pending> waiting;
    std::map<PackKey, std::deque<Pending>> packs;
    size_t packed_waiting = 0;
    std::vector<Pending> pack;  // the pack being solved
    std::unordered_map<uint64_t, Running> running;
    Clock::time_point busy_since{};
    // On an error every query the worker holds completes with it.
    auto held = [&] {
        std::vector<uint64_t> t;
        for (const auto &r : running) t.push_back(r.first);
        for (const Pending &p : pack) t.push_back(p.ticket);
        for (const auto &kv : packs)
            for (const Pending &p : kv.second) t.push_back(p.ticket);
        for (const Pending &p : waiting) t.push_back(p.ticket);
        return t;
    };
    try {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (waiting.empty() && running.empty() && packed_waiting == 0) {
                    if (stop) break;
                    if (inbox.empty()) cv_work.wait_for(lk, std::chrono::milliseconds(20));
                }
                while (!inbox.empty()) {
                    Pending p = inbox.front();
                    inbox.pop_front();
                    if (packable(p.q)) {
                        packs[pack_key(p.q)].push_back(p);
                        ++packed_waiting;
                    } else {
                        waiting.push_back(p);
                    }
                }
                if (stop) {  // destroy drops what was not admitted
                    waiting.clear();
                    packs.clear();
                    packed_waiting = 0;
                }
            }
            // one pack: the key whose oldest query is oldest, up to 8 queries
            if (packed_waiting) {
                if (busy_since == Clock::time_point{}) busy_since = Clock::now();
                auto best = packs.end();
                for (auto it = packs.begin(); it != packs.end(); ++it)
                    if (best == packs.end() || it->second.front().submitted < best->second.front().submitted)
                        best = it;
                pack.clear();
                while (!best->second.empty() && pack.size() < 8) {
                    pack.push_back(best->second.front());
                    best->second.pop_front();
                }
                if (best->second.empty()) packs.erase(best);
                packed_waiting -= pack.size();
                std::vector<hyt_completion> pout;
                run_pack(pack, pout);
                pack.clear();
                const auto now = Clock::now();
                {
                    std::lock_guard<std::mutex> lk(mu);
                    for (const hyt_completion &c : pout) done.push_back(c);
                    st.completed += pout.size();
                    st.packs = packs_run;
                    st.waiting = static_cast<uint32_t>(waiting.size() + inbox.size() + packed_waiting);
                    if (running.empty() && packed_waiting == 0) {
                        st.busy_ms += ms_between(busy_since, now);
                        busy_since = Clock::time_point{};
                    }
                }
                cv_done.notify_all();
            }
            // admit, oldest first
            std::vector<hyt_completion> rejected;
            while (!waiting.empty() && engine->running() < max_running) {
                const Pending &p = waiting.front();
                if (engine->admit(p.q, p.ticket) < 0) {
                    if (engine->slots_in_use() > 0) break;  // wait for running queries to free state
                    hyt_completion c{};                     // does not fit even an idle engine
                    c.ticket = p.ticket;
                    c.status = HYT_E_OOM;
                    c.latency_ms = ms_between(p.submitted, Clock::now());
                    rejected.push_back(c);
                    waiting.pop_front();
                    continue;
                }
                running[p.ticket] = Running{p.submitted, Clock::now()};
                waiting.pop_front();
            }
            if (!rejected.empty()) {
                std::lock_guard<std::mutex> lk(mu);
                for (const hyt_completion &c : rejected) done.push_back(c);
                st.completed += rejected.size();
                cv_done.notify_all();
            }
            if (running.empty()) continue;
            if (busy_since == Clock::time_point{}) busy_since = Clock::now();
            engine->step();
            const auto fin = engine->finished();  // synchronises the stream
            std::vector<hyt_completion> out;
            out.reserve(fin.size());
            for (const auto &f : fin) {
                hyt_completion c{};
                c.ticket = f.second;
                c.status = HYT_OK;
                engine->retire(f.first, &c.result);
                out.push_back(c);
            }
            if (!fin.empty()) HYT_CUDA(cudaStreamSynchronize(stream));  // results are in `out`
            const auto now = Clock::now();
            {
                std::lock_guard<std::mutex> lk(mu);
                ++st.supersteps;
                ++st.graph_launches;
                for (hyt_completion &c : out) {
                    const Running r = running[c.ticket];
                    running.erase(c.ticket);
                    c.queue_ms = ms_between(r.submitted, r.admitted);
                    c.latency_ms = ms_between(r.submitted, now);
                    done.push_back(c);
                    ++st.completed;
                }
                st.running = static_cast<uint32_t>(running.size());
                st.waiting = static_cast<uint32_t>(waiting.size() + inbox.size());
                st.max_running = std::max<uint32_t>(st.max_running, st.running + static_cast<uint32_t>(out.size()));
                st.state_bytes = engine->bytes_in_use();
                st.peak_state_bytes = std::max(st.peak_state_bytes, st.state_bytes);
                if (running.empty() && packed_waiting == 0) {
                    st.busy_ms += ms_between(busy_since, now);
                    busy_since = Clock::time_point{};
                }
            }
            if (!out.empty()) cv_done.notify_all();
        }
    } catch (const Error &e) {
        fail_all(held(), e.code, e.what());
    } catch (const std::exception &e) {
        fail_all(held(), HYT_E_INTERNAL, e.what());
    }
}

// The worker stopped on an error: every query it held completes with it
// (and later submissions are refused).
void ServerImpl::fail_all(const std::vector<uint64_t> &tickets, int code, const char *msg) {
    std::lock_guard<std::mutex> lk(mu);
    failure = code;
    failure_msg = msg;
    for (const uint64_t t : tickets) {
        hyt_completion c{};
        c.ticket = t;
        c.status = code;
        done.push_back(c);
    }
    for (const Pending &p : inbox) {
        hyt_completion c{};
        c.ticket = p.ticket;
        c.status = code;
        done.push_back(c);
    }
    inbox.clear();
    cv_done.notify_all();
}

}  // namespace hyt

struct hyt_server {
    hyt::ServerImpl impl;
};

using namespace hyt;

extern "C" {

int hyt_server_create(hyt_graph *const *graphs, uint32_t num_graphs, const hyt_server_options *options,
                      hyt_server **out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        *out = nullptr;
        if (!graphs || num_graphs == 0) fail(HYT_E_INVALID, "a server needs at least one graph");
        hyt_server_options o = options_or_default(options);
        o.device = resolve_device(o.device);
        auto sv = std::make_unique<hyt_server>();
        ServerImpl &s = sv->impl;
        s.device = o.device;
        for (uint32_t i = 0; i < num_graphs; ++i) {
            if (!graphs[i]) fail(HYT_E_INVALID, "graph handle is NULL");
            if (graphs[i]->impl.device != o.device) fail(HYT_E_INVALID, "every graph must live on the server's device");
            s.graphs.push_back(&graphs[i]->impl);
            graph_vertex_map(graphs[i]->impl);  // queries map their sources on the host
        }
        HYT_CUDA(cudaSetDevice(o.device));
        HYT_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        try {
            s.engine = std::make_unique<QueryEngine>(o.device, s.stream,
                                                     o.state_budget_bytes ? o.state_budget_bytes : (uint64_t(16) << 30));
        } catch (...) {
            cudaStreamDestroy(s.stream);
            throw;
        }
        s.engine->set_graphs(s.graphs);
        BatchTuning t;
        t.delta_mult = o.tuning.delta_mult;
        if (o.tuning.hub_degree) t.hub_degree = o.tuning.hub_degree;
        t.ctas_per_sm = o.tuning.ctas_per_sm;
        s.engine->set_tuning(t);
        s.max_running = o.max_running ? o.max_running : 4096u;
        if (o.pack_min_edges) s.pack_min_edges = o.pack_min_edges == 0xFFFFFFFFu ? ~uint64_t(0) : o.pack_min_edges;
        s.worker = std::thread([&s] { s.loop(); });
        *out = sv.release();
    });
}

int hyt_server_submit(hyt_server *sv, const hyt_query *q, uint64_t *ticket) {
    return guarded([&] {
        if (!sv || !q) fail(HYT_E_INVALID, "NULL argument");
        ServerImpl &s = sv->impl;
        s.engine->validate(*q);
        std::lock_guard<std::mutex> lk(s.mu);
        if (s.failure != HYT_OK) fail(s.failure, "server stopped after an error: " + s.failure_msg);
        if (s.stop) fail(HYT_E_INVALID, "server is shutting down");
        const uint64_t t = s.next_ticket++;
        s.inbox.push_back(ServerImpl::Pending{*q, t, std::chrono::steady_clock::now()});
        ++s.st.submitted;
        if (ticket) *ticket = t;
        s.cv_work.notify_one();
    });
}

int hyt_server_poll(hyt_server *sv, hyt_completion *out, uint32_t max, uint32_t *count, uint32_t wait_ms) {
    return guarded([&] {
        if (!sv || (!out && max) || !count) fail(HYT_E_INVALID, "NULL argument");
        ServerImpl &s = sv->impl;
        std::unique_lock<std::mutex> lk(s.mu);
        if (s.done.empty() && wait_ms)
            s.cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s.done.empty(); });
        uint32_t n = 0;
        while (n < max && !s.done.empty()) {
            out[n++] = s.done.front();
            s.done.pop_front();
        }
        *count = n;
    });
}

int hyt_server_get_stats(hyt_server *sv, hyt_server_stats *stats) {
    return guarded([&] {
        if (!sv || !stats) fail(HYT_E_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(sv->impl.mu);
        *stats = sv->impl.st;
    });
}

int hyt_server_destroy(hyt_server *sv) {
    return guarded([&] {
        if (!sv) return;
        ServerImpl &s = sv->impl;
        {
            std::lock_guard<std::mutex> lk(s.mu);
            s.stop = true;
        }
        s.cv_work.notify_all();
        if (s.worker.joinable()) s.worker.join();
        cudaSetDevice(s.device);
        s.engine.reset();
        if (s.stream) cudaStreamDestroy(s.stream);
        delete sv;
    });
}

}  // extern "C"
