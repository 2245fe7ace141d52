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
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "host_checks.hpp"
#include "graph.cuh"

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
    void fail_all(const std::unordered_map<uint64_t, Running> &running, int code, const char *msg);
};

void ServerImpl::loop() {
    cudaSetDevice(device);
    std::deque<Pending> waiting;
    std::unordered_map<uint64_t, Running> running;
    Clock::time_point busy_since{};
    try {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (waiting.empty() && running.empty()) {
                    if (stop) break;
                    if (inbox.empty()) cv_work.wait_for(lk, std::chrono::milliseconds(20));
                }
                while (!inbox.empty()) {
                    waiting.push_back(inbox.front());
                    inbox.pop_front();
                }
                if (stop) waiting.clear();  // destroy drops what was not admitted
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
                if (running.empty()) {
                    st.busy_ms += ms_between(busy_since, now);
                    busy_since = Clock::time_point{};
                }
            }
            if (!out.empty()) cv_done.notify_all();
        }
    } catch (const Error &e) {
        fail_all(running, e.code, e.what());
    } catch (const std::exception &e) {
        fail_all(running, HYT_E_INTERNAL, e.what());
    }
}

// The worker stopped on an error: every running query completes with it.
void ServerImpl::fail_all(const std::unordered_map<uint64_t, Running> &running, int code, const char *msg) {
    std::lock_guard<std::mutex> lk(mu);
    failure = code;
    failure_msg = msg;
    for (const auto &r : running) {
        hyt_completion c{};
        c.ticket = r.first;
        c.status = code;
        done.push_back(c);
    }
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
