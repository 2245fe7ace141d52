// Out-of-HBM hybrid-transfer engine (HyTM executed).
//
// The graph's edges stay in pinned, device-mapped host memory; HBM holds
// vertex data, a resident subset of partitions (filling the device budget)
// and staging buffers.  For every partition that a PageRank iteration or an
// SSSP round touches, the engine evaluates the HyTM costs -- formulas (1)-(3)
// and Algorithm 1 of the reference's cost model
// (src/transfer/hytm_cost_model.cpp:454-715) -- with link parameters
// measured at start-up instead of the reference's placeholders (RTT = 1,
// CPU throughput = 1 B/s, include/transfer/hytm_cost_model.hpp:55-66):
//   RTT  = (payload * requests per TLP) / measured pinned H2D bandwidth,
//   T_cpu = measured host gather bandwidth of the engine's threads,
//   zero-copy TLPs scaled by measured H2D / zero-copy read bandwidth.
// and executes the selected engine:
//   resident    -- already in HBM, nothing crosses the link;
//   ExpTM-Filter -- the partition is copied (cudaMemcpyAsync on a copy
//                  stream) into one of two staging slots, piece by piece
//                  when it is larger than a slot; consecutive filter pieces
//                  (<= 4, TaskCombiner's rule) share one copy; the next
//                  copy overlaps the kernels reading the current slot;
//   ExpTM-Compaction -- host threads gather the active rows (ids and
//                  weights) into pinned staging, one copy ships the packed
//                  payload (layout of the reference's CompactedPartition);
//   ImpTM-Zero-Copy -- the kernels read the rows in place over the link.
// Every byte that crosses the link is counted per engine.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "common.cuh"
#include "host_checks.hpp"
#include "graph.cuh"
#include "hybrid.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

constexpr size_t kFilterCombineK = 4;  // consecutive filter partitions per copy

enum Engine : uint32_t { kResident = 0, kFilter = 1, kCompaction = 2, kZeroCopy = 3 };

struct LinkParams {
    double h2d_gbs = 0, zc_gbs = 0, gather_gbs = 0;
};

// HyTM cost arithmetic (reference hytm_cost_model.cpp:486-615 and :649-715);
// d1 = bytes shipped per edge, d2 = index bytes per active vertex.
struct Hytm {
    double alpha = 0.8, beta = 0.4, gamma = 0.625;
    double rtt = 1.0, zc_scale = 1.0, cpu_bps = 1.0;
    uint64_t m = 128, mr = 256, d1 = 4, d2 = 8;

    static uint64_t ceil_div(uint64_t a, uint64_t b) { return a / b + (a % b != 0); }

    uint32_t select(uint64_t total_edges, const PartMetrics &pm) const {
        const uint64_t tlp = m * mr;
        const double f = double(ceil_div(total_edges * d1, tlp)) * rtt;
        const uint64_t cbytes = pm.active_edges * d1 + pm.active_vertices * d2;
        const double c = double(ceil_div(cbytes, tlp)) * rtt + double(cbytes) / cpu_bps;
        const double ratio = total_edges ? double(pm.active_edges) / double(total_edges) : 0.0;
        const double rtt_zc = gamma * rtt + (1.0 - gamma) * ratio * rtt;
        const double z = double(ceil_div(pm.zc_requests + pm.zc_alignment, mr)) * rtt_zc * zc_scale;
        if (c < alpha * f && c < beta * z) return kCompaction;
        if (f < z) return kFilter;
        return kZeroCopy;
    }
};

__global__ void zc_read_kernel(const uint4 *src, size_t n, unsigned long long *sink) {
    unsigned long long acc = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const uint4 v = src[i];
        acc += v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9E3779B97F4A7C15ull) atomicAdd(sink, acc);  // keeps the loads alive
}

__global__ void u32_from_u64_offsets_kernel(const uint64_t *off, uint64_t V, uint32_t *deg) {
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x)
        deg[v] = static_cast<uint32_t>(off[v + 1] - off[v]);
}

template <class F>
void parallel_chunks(unsigned threads, uint64_t n, F &&f) {
    if (threads <= 1 || n < 4096) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t step = (n + threads - 1) / threads;
    for (unsigned t = 0; t < threads; ++t) {
        const uint64_t b = t * step, e = std::min(n, b + step);
        if (b >= e) break;
        th.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto &x : th) x.join();
}

// Device-usable address of host memory; registers pageable memory.
const void *device_alias(const void *p, size_t bytes, std::vector<void *> &registered) {
    if (!p || !bytes) return p;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) (void)cudaGetLastError();
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged)
        fail(HYT_E_INVALID, "hybrid graphs take host arrays (pinned or pageable), not device memory");
    if (at.type != cudaMemoryTypeHost) {
        // pin the enclosing pages (read-only mapping where the platform has it)
        const uintptr_t page = 4096;
        const uintptr_t b = reinterpret_cast<uintptr_t>(p) & ~(page - 1);
        const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes + page - 1) & ~(page - 1);
        void *base = reinterpret_cast<void *>(b);
        cudaError_t r = cudaHostRegister(base, e - b, cudaHostRegisterMapped | cudaHostRegisterReadOnly);
        if (r != cudaSuccess && r != cudaErrorHostMemoryAlreadyRegistered) {
            (void)cudaGetLastError();
            r = cudaHostRegister(base, e - b, cudaHostRegisterMapped);
        }
        if (r == cudaSuccess) {
            registered.push_back(base);
        } else if (r != cudaErrorHostMemoryAlreadyRegistered) {
            HYT_CUDA(r);
        }
        (void)cudaGetLastError();
    }
    void *d = nullptr;
    HYT_CUDA(cudaHostGetDevicePointer(&d, const_cast<void *>(p), 0));
    return d;
}


// A piece: a vertex range of one partition whose edges are contiguous in the
// CSR (push) or CSC (pull).  A resident partition is one piece; any other is
// cut into pieces of at most one staging slot so that ExpTM-Filter can ship
// it slot by slot.
struct Piece {
    uint32_t part;
    uint32_t v0, v1;
    uint64_t e0, e1;
    PullPart tasks;  // pull side: tiles and long-row chunks of the piece
};

// Consecutive filter pieces shipped by one copy (TaskCombiner's rule: at
// most kFilterCombineK of them, and they must fit one slot).
struct Group {
    size_t first, last;  // pieces [first, last)
    uint64_t e0, e1;
};

}  // namespace

struct HybridImpl {
    GraphImpl g;  // vertex data on the device; edges are not held here
    cudaStream_t copy = nullptr;
    uint32_t part_shift = 20;
    size_t P = 0;
    uint32_t flags = 0;
    unsigned threads = 1;
    uint64_t budget = 0;
    uint32_t force = 0;

    // host arrays and their device-usable aliases
    const uint64_t *h_off = nullptr, *h_in_off = nullptr;
    const uint32_t *h_cols = nullptr, *h_w = nullptr, *h_in_src = nullptr;
    const uint32_t *z_cols = nullptr, *z_w = nullptr, *z_in_src = nullptr;
    std::vector<void *> registered;

    // partition geometry: [e0, e1) of the CSR (push) and CSC (pull)
    std::vector<uint64_t> push_e0, push_e1, pull_e0, pull_e1;
    std::vector<Piece> push_pieces, pull_pieces;
    std::vector<size_t> push_first, pull_first;  // first piece of each partition, [P + 1]
    std::vector<uint64_t> pull_zc_bytes;          // 128-byte lines of each partition's CSC
    std::vector<PartMetrics> pull_metrics;        // all vertices active

    // residency
    std::vector<uint8_t> push_res, pull_res;
    std::vector<uint64_t> push_res_pos, pull_res_pos;
    DeviceArray<uint32_t> push_res_cols, push_res_w, pull_res_src;
    uint64_t resident_bytes = 0;

    // staging: two slots, shared by both sides
    DeviceArray<uint32_t> stage_a[2], stage_b[2];  // push: cols / weights; pull: ids in stage_a
    uint64_t stage_edges = 0;
    cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};

    // compaction staging
    DeviceArray<unsigned char> cdev;
    PinnedArray<unsigned char> chost;
    uint64_t cbytes = 0;

    LinkParams link;
    Hytm model;
    hyt_hybrid_stats stats{};

    ~HybridImpl() {
        for (int i = 0; i < 2; ++i) {
            if (ev_ready[i]) cudaEventDestroy(ev_ready[i]);
            if (ev_free[i]) cudaEventDestroy(ev_free[i]);
        }
        if (copy) cudaStreamDestroy(copy);
        for (void *p : registered) cudaHostUnregister(p);
        if (g.own_stream && g.stream) cudaStreamDestroy(g.stream);
    }

    uint64_t push_bytes_per_edge() const { return h_w ? 8 : 4; }

    // Copies edges [e0, e1) of one side into slot `slot` on the copy stream,
    // once the slot's previous readers are done.
    void issue_copy(bool push_side, int slot, uint64_t e0, uint64_t e1) {
        HYT_CUDA(cudaStreamWaitEvent(copy, ev_free[slot], 0));
        const uint64_t n = e1 - e0;
        const uint32_t *a = push_side ? h_cols : h_in_src;
        HYT_CUDA(cudaMemcpyAsync(stage_a[slot].get(), a + e0, n * 4, cudaMemcpyHostToDevice, copy));
        stats.filter_bytes += n * 4;
        if (push_side && h_w) {
            HYT_CUDA(cudaMemcpyAsync(stage_b[slot].get(), h_w + e0, n * 4, cudaMemcpyHostToDevice, copy));
            stats.filter_bytes += n * 4;
        }
        HYT_CUDA(cudaEventRecord(ev_ready[slot], copy));
        ++stats.copies;
    }
};

namespace {

void measure_link(HybridImpl &h) {
    cudaStream_t s = h.g.stream;
    const size_t bytes = size_t(256) << 20;
    PinnedArray<unsigned char> hb(bytes, cudaHostAllocMapped);
    std::memset(hb.ptr, 1, bytes);
    DeviceArray<unsigned char> db(bytes);
    DeviceArray<unsigned long long> sink(1);
    EventTimer t;
    double best = 1e30, best_zc = 1e30;
    void *zp = nullptr;
    HYT_CUDA(cudaHostGetDevicePointer(&zp, hb.ptr, 0));
    for (int r = 0; r < 3; ++r) {
        t.start(s);
        HYT_CUDA(cudaMemcpyAsync(db.get(), hb.ptr, bytes, cudaMemcpyHostToDevice, s));
        t.stop(s);
        best = std::min(best, t.ms());
        t.start(s);
        zc_read_kernel<<<sm_count() * 8, 256, 0, s>>>(static_cast<const uint4 *>(zp), bytes / 16, sink.get());
        t.stop(s);
        HYT_CUDA(cudaGetLastError());
        best_zc = std::min(best_zc, t.ms());
    }
    h.link.h2d_gbs = bytes / (best * 1e-3) / 1e9;
    h.link.zc_gbs = bytes / (best_zc * 1e-3) / 1e9;
    // host gather bandwidth: random 256-edge rows of the graph's own ids
    const uint32_t *src = h.h_cols ? h.h_cols : h.h_in_src;
    const uint64_t E = h.g.E;
    if (src && E > 4096) {
        const uint64_t rows = 1 << 15, len = 256;
        std::vector<uint32_t> out(rows * len);
        const auto t0 = std::chrono::steady_clock::now();
        parallel_chunks(h.threads, rows, [&](uint64_t b, uint64_t e) {
            uint64_t x = 0x9E3779B97F4A7C15ull * (b + 1);
            for (uint64_t r = b; r < e; ++r) {
                x ^= x >> 12;
                x ^= x << 25;
                x ^= x >> 27;
                const uint64_t at = (x * 0x2545F4914F6CDD1Dull) % (E - len);
                std::memcpy(&out[r * len], src + at, len * 4);
            }
        });
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        h.link.gather_gbs = rows * len * 4 / std::max(sec, 1e-6) / 1e9;
    } else {
        h.link.gather_gbs = 1.0;
    }
    h.model.rtt = double(h.model.m * h.model.mr) / (h.link.h2d_gbs * 1e9);
    h.model.zc_scale = h.link.h2d_gbs / std::max(h.link.zc_gbs, 1e-3);
    h.model.cpu_bps = h.link.gather_gbs * 1e9;
}

// Staging slot size (bytes) for a side's budget: an eighth of it, between
// 1 MiB and 1 GiB (copies of 1 GiB already run at the link's peak).
uint64_t slot_bytes_for(uint64_t side_budget) {
    return std::min<uint64_t>(std::max<uint64_t>(side_budget / 8, uint64_t(1) << 20), uint64_t(1) << 30);
}

// Greedy residency: after the staging reserve, the largest partitions first
// while they fit.  Every resident partition is one contiguous run of the
// resident array, in partition order.
void choose_residency(const std::vector<uint64_t> &e0, const std::vector<uint64_t> &e1, uint64_t bpe,
                      uint64_t budget, std::vector<uint8_t> &res, std::vector<uint64_t> &pos, uint64_t &used_edges) {
    const size_t P = e0.size();
    std::vector<size_t> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return e1[a] - e0[a] > e1[b] - e0[b]; });
    res.assign(P, 0);
    pos.assign(P, 0);
    uint64_t used = 0;
    for (size_t p : order) {
        const uint64_t n = e1[p] - e0[p];
        if (n && (used + n) * bpe <= budget) {
            res[p] = 1;
            used += n;
        }
    }
    used_edges = 0;
    for (size_t p = 0; p < P; ++p)
        if (res[p]) {
            pos[p] = used_edges;
            used_edges += e1[p] - e0[p];
        }
}

void upload_resident(HybridImpl &h, const std::vector<uint8_t> &res, const std::vector<uint64_t> &e0,
                     const std::vector<uint64_t> &e1, const std::vector<uint64_t> &pos, const uint32_t *ha,
                     const uint32_t *hb, uint32_t *da, uint32_t *db) {
    for (size_t p = 0; p < res.size(); ++p) {
        if (!res[p]) continue;
        const uint64_t n = e1[p] - e0[p];
        HYT_CUDA(cudaMemcpyAsync(da + pos[p], ha + e0[p], n * 4, cudaMemcpyHostToDevice, h.g.stream));
        if (hb) HYT_CUDA(cudaMemcpyAsync(db + pos[p], hb + e0[p], n * 4, cudaMemcpyHostToDevice, h.g.stream));
    }
    HYT_CUDA(cudaStreamSynchronize(h.g.stream));
}

// Push pieces: non-resident partitions cut at vertex boundaries so that a
// piece holds at most `cap` edges (a single larger row is a piece alone).
void build_push_pieces(HybridImpl &h, uint64_t cap) {
    h.push_pieces.clear();
    h.push_first.assign(h.P + 1, 0);
    for (size_t p = 0; p < h.P; ++p) {
        h.push_first[p] = h.push_pieces.size();
        const uint64_t v0 = uint64_t(p) << h.part_shift;
        const uint64_t v1 = std::min<uint64_t>(h.g.V, (uint64_t(p) + 1) << h.part_shift);
        if (h.push_res[p] || h.push_e1[p] - h.push_e0[p] <= cap) {
            h.push_pieces.push_back(Piece{static_cast<uint32_t>(p), static_cast<uint32_t>(v0),
                                          static_cast<uint32_t>(v1), h.push_e0[p], h.push_e1[p], PullPart{}});
            continue;
        }
        uint64_t a = v0;
        while (a < v1) {
            uint64_t b = a + 1;
            while (b < v1 && h.h_off[b + 1] - h.h_off[a] <= cap) ++b;
            h.push_pieces.push_back(Piece{static_cast<uint32_t>(p), static_cast<uint32_t>(a),
                                          static_cast<uint32_t>(b), h.h_off[a], h.h_off[b], PullPart{}});
            a = b;
        }
    }
    h.push_first[h.P] = h.push_pieces.size();
}

// Pull pieces: tiles are first split at partition boundaries (no tile
// straddles two partitions); non-resident partitions are then cut between
// tiles so that a piece holds at most `cap` in-edges.  A long row's chunk
// tasks belong to the piece of the tile it ends.
void build_pull_pieces(HybridImpl &h, uint64_t cap) {
    GraphImpl &g = h.g;
    cudaStream_t s = g.stream;
    std::vector<uint32_t> ts(g.num_tiles + 1);
    HYT_CUDA(cudaMemcpyAsync(ts.data(), g.tile_start.get(), ts.size() * 4, cudaMemcpyDeviceToHost, s));
    std::vector<LongRow> lr(g.num_long);
    if (g.num_long)
        HYT_CUDA(cudaMemcpyAsync(lr.data(), g.long_rows.get(), lr.size() * sizeof(LongRow), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> bounds;
    bounds.reserve(ts.size() + h.P + 1);
    for (uint32_t v : ts) bounds.push_back(v);
    for (size_t p = 0; p <= h.P; ++p)
        bounds.push_back(static_cast<uint32_t>(std::min<uint64_t>(g.V, uint64_t(p) << h.part_shift)));
    std::sort(bounds.begin(), bounds.end());
    bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
    g.num_tiles = bounds.size() - 1;
    g.tile_start.allocate(bounds.size());
    HYT_CUDA(cudaMemcpyAsync(g.tile_start.get(), bounds.data(), bounds.size() * 4, cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));

    const uint64_t *off = h.h_in_off;
    h.pull_pieces.clear();
    h.pull_first.assign(h.P + 1, 0);
    uint64_t t = 0, c = 0, li = 0;
    auto close_piece = [&](size_t p, uint64_t t0, uint64_t t1, uint64_t c0) {
        const uint32_t va = bounds[t0], vb = bounds[t1];
        while (li < g.num_long && lr[li].row < vb) {
            c = lr[li].first_chunk + lr[li].num_chunks;
            ++li;
        }
        h.pull_pieces.push_back(Piece{static_cast<uint32_t>(p), va, vb, off[va], off[vb], PullPart{c0, c, t0, t1}});
    };
    for (size_t p = 0; p < h.P; ++p) {
        h.pull_first[p] = h.pull_pieces.size();
        const uint64_t v1 = std::min<uint64_t>(g.V, (uint64_t(p) + 1) << h.part_shift);
        const uint64_t tb = t;
        while (t < g.num_tiles && bounds[t] < v1) ++t;
        const uint64_t te = t;
        if (h.pull_res[p] || h.pull_e1[p] - h.pull_e0[p] <= cap) {
            close_piece(p, tb, te, c);
            continue;
        }
        uint64_t a = tb;
        while (a < te) {
            uint64_t b = a + 1;
            while (b < te && off[bounds[b + 1]] - off[bounds[a]] <= cap) ++b;
            close_piece(p, a, b, c);
            a = b;
        }
    }
    h.pull_first[h.P] = h.pull_pieces.size();
}

// Groups consecutive pieces whose partitions chose ExpTM-Filter.
std::vector<Group> filter_groups(const std::vector<Piece> &pieces, const std::vector<uint32_t> &engine,
                                 uint64_t slot_edges) {
    std::vector<Group> out;
    for (size_t i = 0; i < pieces.size();) {
        if (engine[pieces[i].part] != kFilter) {
            ++i;
            continue;
        }
        Group gr{i, i, pieces[i].e0, pieces[i].e0};
        while (i < pieces.size() && engine[pieces[i].part] == kFilter && gr.last - gr.first < kFilterCombineK &&
               pieces[i].e0 == gr.e1 && pieces[i].e1 - gr.e0 <= slot_edges) {
            gr.e1 = pieces[i].e1;
            gr.last = ++i;
        }
        out.push_back(gr);
    }
    return out;
}

// A partition may use ExpTM-Filter only if each of its pieces fits a slot.
bool filterable(const std::vector<Piece> &pieces, const std::vector<size_t> &first, size_t p, uint64_t slot_edges) {
    if (first[p] == first[p + 1]) return false;
    for (size_t i = first[p]; i < first[p + 1]; ++i)
        if (pieces[i].e1 - pieces[i].e0 > slot_edges) return false;
    return true;
}

// ------------------------------------------------------------ push source --
class HybridPush final : public PushSource {
public:
    explicit HybridPush(HybridImpl &h) : h_(h) {}
    uint32_t part_shift() const override { return h_.part_shift; }
    size_t parts() const override { return h_.P; }

    void plan_round(const std::vector<PartMetrics> &m, RoundPlan &plan) override {
        const size_t P = h_.P;
        const uint64_t bpe = h_.push_bytes_per_edge();
        engines_.assign(P, kZeroCopy);
        std::vector<EdgeLoc> base(P);
        for (size_t p = 0; p < P; ++p) base[p] = EdgeLoc{h_.z_cols, h_.z_w, kLocDirect, 0u, 0xFFFFFFFFu, 0u};
        uint64_t cpay = 0;
        for (size_t p = 0; p < P; ++p) {
            if (h_.push_res[p]) {
                engines_[p] = kResident;
                base[p].cols = h_.push_res_cols.get() + h_.push_res_pos[p] - h_.push_e0[p];
                base[p].weights = h_.push_res_w.get() ? h_.push_res_w.get() + h_.push_res_pos[p] - h_.push_e0[p]
                                                      : nullptr;
                continue;
            }
            if (m[p].active_vertices == 0) continue;  // nothing to read this round
            uint32_t e = h_.force ? h_.force : h_.model.select(h_.push_e1[p] - h_.push_e0[p], m[p]);
            if (e == kFilter && !filterable(h_.push_pieces, h_.push_first, p, h_.stage_edges)) e = kZeroCopy;
            if (e == kCompaction) {
                const uint64_t need = m[p].active_edges * bpe + m[p].active_vertices * 12 + 64;
                if (cpay + need > h_.cbytes) {
                    e = kZeroCopy;
                } else {
                    cpay += need;
                }
            }
            engines_[p] = e;
            if (e == kCompaction) base[p].mode = kLocCompacted;
        }
        // wave 0: resident, zero-copy and compacted partitions; then one wave
        // per filter group, with the window of each partition's pieces in it
        groups_ = filter_groups(h_.push_pieces, engines_, h_.stage_edges);
        plan.compacted = false;
        for (size_t p = 0; p < P; ++p) plan.compacted |= engines_[p] == kCompaction;
        plan.waves.assign(1 + groups_.size(), base);
        for (size_t p = 0; p < P; ++p)
            if (engines_[p] == kFilter) plan.waves[0][p].mode = kLocSkip;
        for (size_t w = 0; w < groups_.size(); ++w) {
            auto &wl = plan.waves[w + 1];
            const Group &gr = groups_[w];
            const int slot = static_cast<int>(w & 1);
            for (size_t p = 0; p < P; ++p)
                if (wl[p].mode != kLocCompacted) wl[p].mode = kLocSkip;
            for (size_t i = gr.first; i < gr.last; ++i) {
                const Piece &pc = h_.push_pieces[i];
                EdgeLoc &L = wl[pc.part];
                if (L.mode == kLocSkip) {
                    L = EdgeLoc{h_.stage_a[slot].get() - gr.e0, h_.z_w ? h_.stage_b[slot].get() - gr.e0 : nullptr,
                                kLocDirect, pc.v0, pc.v1, 0u};
                } else {
                    L.vhi = pc.v1;  // pieces of a partition in one group are consecutive
                }
            }
        }
        for (size_t p = 0; p < P; ++p) {
            if (!m[p].active_vertices) continue;
            switch (engines_[p]) {
                case kResident: ++h_.stats.resident_decisions; break;
                case kFilter: ++h_.stats.filter_decisions; break;
                case kCompaction: ++h_.stats.compaction_decisions; break;
                default:
                    ++h_.stats.zero_copy_decisions;
                    // 128-byte lines of the ids (and weights) the kernels touch
                    h_.stats.zero_copy_bytes += (m[p].zc_requests + m[p].zc_alignment) * 128 * (h_.z_w ? 2 : 1);
            }
            if (engines_[p] != kResident) h_.stats.necessary_bytes += m[p].active_edges * bpe;
        }
        for (size_t w = 0; w < std::min<size_t>(2, groups_.size()); ++w) issue(w);
    }

    void enter_wave(size_t w, cudaStream_t s) override {
        if (w == 0) return;
        HYT_CUDA(cudaStreamWaitEvent(s, h_.ev_ready[(w - 1) & 1], 0));
    }

    void leave_wave(size_t w, cudaStream_t s) override {
        if (w == 0) return;
        const size_t gi = w - 1;
        HYT_CUDA(cudaEventRecord(h_.ev_free[gi & 1], s));
        if (gi + 2 < groups_.size()) issue(gi + 2);
    }

    CompactPayload compact(const uint32_t *verts, uint64_t n, cudaStream_t s) override {
        // host threads: row lengths, prefix, then the packed rows
        const uint64_t *off = h_.h_off;
        std::vector<uint64_t> index(n + 1, 0);
        for (uint64_t i = 0; i < n; ++i) index[i + 1] = index[i] + (off[verts[i] + 1] - off[verts[i]]);
        const uint64_t edges = index[n];
        const uint64_t bpe = h_.push_bytes_per_edge();
        // pinned layout: verts u32[n] | index u64[n+1] | cols u32[edges] | weights u32[edges]
        const uint64_t o_idx = (uint64_t(n) * 4 + 15) & ~15ull;
        const uint64_t o_cols = (o_idx + (n + 1) * 8 + 15) & ~15ull;
        const uint64_t o_w = (o_cols + edges * 4 + 15) & ~15ull;
        const uint64_t total = o_w + (bpe == 8 ? edges * 4 : 0);
        if (total > h_.cbytes) fail(HYT_E_INTERNAL, "compaction payload exceeds its staging buffer");
        unsigned char *hb = h_.chost.ptr;
        const auto t0 = std::chrono::steady_clock::now();
        std::memcpy(hb, verts, n * 4);
        std::memcpy(hb + o_idx, index.data(), (n + 1) * 8);
        uint32_t *hc = reinterpret_cast<uint32_t *>(hb + o_cols);
        uint32_t *hw = reinterpret_cast<uint32_t *>(hb + o_w);
        parallel_chunks(h_.threads, n, [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i) {
                const uint64_t r0 = off[verts[i]], len = index[i + 1] - index[i];
                std::memcpy(hc + index[i], h_.h_cols + r0, len * 4);
                if (bpe == 8) std::memcpy(hw + index[i], h_.h_w + r0, len * 4);
            }
        });
        h_.stats.compaction_host_ms +=
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        HYT_CUDA(cudaMemcpyAsync(h_.cdev.get(), hb, total, cudaMemcpyHostToDevice, s));
        h_.stats.compaction_bytes += total;
        CompactPayload pk{};
        pk.verts = reinterpret_cast<const uint32_t *>(h_.cdev.get());
        pk.index = reinterpret_cast<const uint64_t *>(h_.cdev.get() + o_idx);
        pk.cols = reinterpret_cast<const uint32_t *>(h_.cdev.get() + o_cols);
        pk.weights = bpe == 8 ? reinterpret_cast<const uint32_t *>(h_.cdev.get() + o_w) : nullptr;
        pk.rows = n;
        pending_ = true;  // the buffers are reused next round
        return pk;
    }

    void end_round(cudaStream_t s) override {
        ++h_.stats.rounds;
        if (pending_) {
            HYT_CUDA(cudaStreamSynchronize(s));
            pending_ = false;
        }
    }

private:
    void issue(size_t gi) {
        h_.issue_copy(true, static_cast<int>(gi & 1), groups_[gi].e0, groups_[gi].e1);
    }

    HybridImpl &h_;
    std::vector<uint32_t> engines_;
    std::vector<Group> groups_;
    bool pending_ = false;
};

// ------------------------------------------------------------ pull source --
class HybridPull final : public PullSource {
public:
    // Every vertex is active in every PageRank iteration, so each
    // partition's decision is the same every iteration: it is taken once
    // per solve from metrics over the partition's whole CSC.
    explicit HybridPull(HybridImpl &h) : h_(h) {
        const size_t P = h_.P;
        engines_.assign(P, kZeroCopy);
        for (size_t p = 0; p < P; ++p) {
            const uint64_t n = h_.pull_e1[p] - h_.pull_e0[p];
            if (h_.pull_res[p]) {
                engines_[p] = kResident;
                continue;
            }
            if (n == 0) continue;
            uint32_t e = h_.force ? h_.force : h_.model.select(n, h_.pull_metrics[p]);
            if (e == kCompaction) e = kFilter;  // all rows active: the packed payload is the partition
            if (e == kFilter && !filterable(h_.pull_pieces, h_.pull_first, p, h_.stage_edges)) e = kZeroCopy;
            engines_[p] = e;
            if (e == kZeroCopy) zc_bytes_ += h_.pull_zc_bytes[p];
        }
        groups_ = filter_groups(h_.pull_pieces, engines_, h_.stage_edges);
        group_of_.assign(h_.pull_pieces.size(), kNone);
        for (size_t gi = 0; gi < groups_.size(); ++gi)
            for (size_t i = groups_[gi].first; i < groups_[gi].last; ++i) group_of_[i] = gi;
    }

    size_t parts() const override { return h_.pull_pieces.size(); }
    PullPart part(size_t i) const override { return h_.pull_pieces[i].tasks; }

    void begin_iteration(cudaStream_t) override {
        for (size_t gi = 0; gi < std::min<size_t>(2, groups_.size()); ++gi) issue(gi);
        for (size_t p = 0; p < h_.P; ++p) {
            if (h_.pull_e1[p] == h_.pull_e0[p]) continue;
            switch (engines_[p]) {
                case kResident: ++h_.stats.resident_decisions; break;
                case kFilter: ++h_.stats.filter_decisions; break;
                default: ++h_.stats.zero_copy_decisions;
            }
            if (engines_[p] != kResident) h_.stats.necessary_bytes += (h_.pull_e1[p] - h_.pull_e0[p]) * 4;
        }
        h_.stats.zero_copy_bytes += zc_bytes_;
        ++h_.stats.rounds;
    }

    const uint32_t *acquire(size_t i, cudaStream_t s) override {
        const Piece &pc = h_.pull_pieces[i];
        switch (engines_[pc.part]) {
            case kResident: return h_.pull_res_src.get() + h_.pull_res_pos[pc.part] - h_.pull_e0[pc.part];
            case kFilter: {
                const size_t gi = group_of_[i];
                if (i == groups_[gi].first) HYT_CUDA(cudaStreamWaitEvent(s, h_.ev_ready[gi & 1], 0));
                return h_.stage_a[gi & 1].get() - groups_[gi].e0;
            }
            default: return h_.z_in_src;
        }
    }

    void release(size_t i, cudaStream_t s) override {
        const size_t gi = group_of_[i];
        if (gi == kNone || i + 1 != groups_[gi].last) return;
        HYT_CUDA(cudaEventRecord(h_.ev_free[gi & 1], s));
        if (gi + 2 < groups_.size()) issue(gi + 2);
    }

private:
    static constexpr size_t kNone = ~size_t(0);

    void issue(size_t gi) { h_.issue_copy(false, static_cast<int>(gi & 1), groups_[gi].e0, groups_[gi].e1); }

    HybridImpl &h_;
    std::vector<uint32_t> engines_;
    std::vector<Group> groups_;
    std::vector<size_t> group_of_;
    uint64_t zc_bytes_ = 0;
};

HybridImpl *impl(hyt_hybrid *x) {
    if (!x) fail(HYT_E_INVALID, "hybrid handle is NULL");
    return reinterpret_cast<HybridImpl *>(x);
}

}  // namespace

// --------------------------------------------------------------- create ----
HybridImpl *hybrid_create(const hyt_csr *csr, const hyt_csc *csc, const hyt_hybrid_options &o) {
    auto h = std::make_unique<HybridImpl>();
    GraphImpl &g = h->g;
    g.device = resolve_device(o.device);
    HYT_CUDA(cudaSetDevice(g.device));
    HYT_CUDA(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    g.own_stream = true;
    g.host_scratch.allocate(64);
    HYT_CUDA(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        HYT_CUDA(cudaEventCreateWithFlags(&h->ev_ready[i], cudaEventDisableTiming));
        HYT_CUDA(cudaEventCreateWithFlags(&h->ev_free[i], cudaEventDisableTiming));
    }
    const uint32_t pv = o.partition_vertices ? o.partition_vertices : (1u << 20);
    if (pv & (pv - 1)) fail(HYT_E_INVALID, "partition_vertices must be a power of two");
    h->part_shift = 0;
    while ((1u << h->part_shift) < pv) ++h->part_shift;
    h->flags = o.flags ? o.flags : HYT_GRAPH_ALL;
    h->budget = o.device_budget_bytes ? o.device_budget_bytes : (8ull << 30);
    h->threads = o.host_threads ? o.host_threads : std::max(1u, std::thread::hardware_concurrency());
    h->force = o.force_engine;
    if (h->force > kZeroCopy) fail(HYT_E_INVALID, "force_engine must be 0..3");
    if (o.alpha > 0) h->model.alpha = o.alpha;
    if (o.beta > 0) h->model.beta = o.beta;
    if (o.gamma > 0) h->model.gamma = o.gamma;

    const bool push = h->flags & HYT_GRAPH_PUSH, pull = h->flags & HYT_GRAPH_PULL;
    if (!csr) fail(HYT_E_INVALID, "csr is NULL");
    if (pull && !csc) fail(HYT_E_INVALID, "HYT_GRAPH_PULL needs the CSC (hyt_csc)");
    const uint64_t V = csr->num_vertices, E = csr->num_edges;
    if (V == 0 || V > 0x7FFFFFFFull) fail(HYT_E_INVALID, "hybrid graphs hold 1 .. 2^31-1 vertices");
    if (csr->weight_kind == HYT_WEIGHTS_F32) fail(HYT_E_UNSUPPORTED, "hybrid graphs take uint32 or no weights");
    if (pull && (csc->num_vertices != V || csc->num_edges != E)) fail(HYT_E_INVALID, "CSC does not match the CSR");
    g.V = V;
    g.E = E;
    g.flags = h->flags;
    g.weight_kind = csr->weight_kind;
    h->P = static_cast<size_t>((V + (uint64_t(1) << h->part_shift) - 1) >> h->part_shift);
    if (h->P > 1024) fail(HYT_E_UNSUPPORTED, "at most 1024 partitions (raise partition_vertices)");

    h->h_off = csr->row_offsets;
    h->h_cols = csr->column_indices;
    h->h_w = csr->weight_kind == HYT_WEIGHTS_U32 ? static_cast<const uint32_t *>(csr->weights) : nullptr;
    if (is_device_pointer(h->h_off) || is_device_pointer(h->h_cols))
        fail(HYT_E_INVALID, "hybrid graphs take host arrays, not device memory");
    if (h->h_off[0] != 0 || h->h_off[V] != E) fail(HYT_E_INVALID, "row offsets must start at 0 and end at E");

    // vertex data on the device
    g.row_offsets.allocate(V + 1);
    HYT_CUDA(cudaMemcpyAsync(g.row_offsets.get(), h->h_off, (V + 1) * 8, cudaMemcpyHostToDevice, g.stream));
    g.out_degree.allocate(V);
    u32_from_u64_offsets_kernel<<<grid_for(V, 256), 256, 0, g.stream>>>(g.row_offsets.get(), V, g.out_degree.get());
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaStreamSynchronize(g.stream));

    // partition geometry
    h->push_e0.resize(h->P);
    h->push_e1.resize(h->P);
    for (size_t p = 0; p < h->P; ++p) {
        h->push_e0[p] = h->h_off[std::min<uint64_t>(V, uint64_t(p) << h->part_shift)];
        h->push_e1[p] = h->h_off[std::min<uint64_t>(V, (uint64_t(p) + 1) << h->part_shift)];
    }
    if (push) {
        h->z_cols = static_cast<const uint32_t *>(device_alias(h->h_cols, E * 4, h->registered));
        if (h->h_w) h->z_w = static_cast<const uint32_t *>(device_alias(h->h_w, E * 4, h->registered));
    }
    if (pull) {
        h->h_in_off = csc->in_offsets;
        h->h_in_src = csc->in_sources;
        if (is_device_pointer(h->h_in_off) || is_device_pointer(h->h_in_src))
            fail(HYT_E_INVALID, "hybrid graphs take host arrays, not device memory");
        if (h->h_in_off[0] != 0 || h->h_in_off[V] != E) fail(HYT_E_INVALID, "CSC offsets must start at 0 and end at E");
        h->z_in_src = static_cast<const uint32_t *>(device_alias(h->h_in_src, E * 4, h->registered));
        h->pull_e0.resize(h->P);
        h->pull_e1.resize(h->P);
        h->pull_zc_bytes.assign(h->P, 0);
        h->pull_metrics.assign(h->P, PartMetrics{});
        for (size_t p = 0; p < h->P; ++p) {
            const uint64_t v0 = std::min<uint64_t>(V, uint64_t(p) << h->part_shift);
            const uint64_t v1 = std::min<uint64_t>(V, (uint64_t(p) + 1) << h->part_shift);
            h->pull_e0[p] = h->h_in_off[v0];
            h->pull_e1[p] = h->h_in_off[v1];
            PartMetrics &pm = h->pull_metrics[p];
            pm.active_vertices = v1 - v0;
            pm.active_edges = h->pull_e1[p] - h->pull_e0[p];
            for (uint64_t v = v0; v < v1; ++v) {
                const uint64_t d = h->h_in_off[v + 1] - h->h_in_off[v];
                if (!d) continue;
                pm.zc_requests += (d * 4 + 127) / 128;
                if ((h->h_in_off[v] * 4) % 128) ++pm.zc_alignment;
            }
            // a tile reads its partition's sources as one contiguous span
            h->pull_zc_bytes[p] = (pm.active_edges * 4 + 127) / 128 * 128;
        }
    }

    // Budget: two staging slots (+ the compaction buffer, half a slot, on
    // the push side), the rest resident; both sides split it when both are
    // built, and share the slots.
    const uint64_t bpe_push = h->h_w ? 8 : 4;
    const uint64_t side_budget = (push && pull) ? h->budget / 2 : h->budget;
    const uint64_t slot = slot_bytes_for(side_budget);
    uint64_t slot_edges = 0;
    if (push) {
        const uint64_t reserve = 2 * slot + slot / 2;
        uint64_t res_edges = 0;
        choose_residency(h->push_e0, h->push_e1, bpe_push, side_budget > reserve ? side_budget - reserve : 0,
                         h->push_res, h->push_res_pos, res_edges);
        build_push_pieces(*h, slot / bpe_push);
        uint64_t need = 0, nonres = 0;  // slots no larger than the largest staged piece
        for (const Piece &pc : h->push_pieces)
            if (!h->push_res[pc.part]) {
                need = std::max(need, std::min(pc.e1 - pc.e0, slot / bpe_push));
                nonres += pc.e1 - pc.e0;
            }
        slot_edges = std::max(slot_edges, need);
        h->cbytes = std::min(slot / 2, nonres * bpe_push + (uint64_t(1) << 16) * 12);
        if (!nonres) h->cbytes = 0;
        h->push_res_cols.allocate(std::max<uint64_t>(res_edges, 1));
        if (h->h_w) h->push_res_w.allocate(std::max<uint64_t>(res_edges, 1));
        upload_resident(*h, h->push_res, h->push_e0, h->push_e1, h->push_res_pos, h->h_cols, h->h_w,
                        h->push_res_cols.get(), h->push_res_w.get());
        h->resident_bytes += res_edges * bpe_push;
    }
    if (pull) {
        const uint64_t reserve = 2 * slot;
        uint64_t res_edges = 0;
        choose_residency(h->pull_e0, h->pull_e1, 4, side_budget > reserve ? side_budget - reserve : 0, h->pull_res,
                         h->pull_res_pos, res_edges);
        g.in_offsets.allocate(V + 1);
        HYT_CUDA(cudaMemcpyAsync(g.in_offsets.get(), h->h_in_off, (V + 1) * 8, cudaMemcpyHostToDevice, g.stream));
        HYT_CUDA(cudaStreamSynchronize(g.stream));
        g.tile_cost = kTileCostDefault;
        g.num_hot = 0;  // host sources are untagged
        build_pull_tiles(g, g.stream);
        build_pull_pieces(*h, slot / 4);
        uint64_t need = 0;
        for (const Piece &pc : h->pull_pieces)
            if (!h->pull_res[pc.part]) need = std::max(need, std::min(pc.e1 - pc.e0, slot / 4));
        slot_edges = std::max(slot_edges, need);
        h->pull_res_src.allocate(std::max<uint64_t>(res_edges, 1));
        upload_resident(*h, h->pull_res, h->pull_e0, h->pull_e1, h->pull_res_pos, h->h_in_src, nullptr,
                        h->pull_res_src.get(), nullptr);
        h->resident_bytes += res_edges * 4;
    }
    h->stage_edges = slot_edges;
    for (int i = 0; i < 2; ++i) {
        if (slot_edges) h->stage_a[i].allocate(slot_edges);
        if (slot_edges && push && h->h_w) h->stage_b[i].allocate(slot_edges);
        HYT_CUDA(cudaEventRecord(h->ev_free[i], g.stream));
    }
    if (h->cbytes) {
        h->cdev.allocate(h->cbytes);
        h->chost.allocate(h->cbytes);
    }
    measure_link(*h);
    return h.release();
}

}  // namespace hyt

using namespace hyt;

extern "C" {

int hyt_hybrid_create(const hyt_csr *csr, const hyt_csc *csc, const hyt_hybrid_options *options,
                      hyt_hybrid **out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        *out = nullptr;
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            (void)cudaGetLastError();
            fail(HYT_E_NO_DEVICE, "no CUDA device is available");
        }
        hyt_hybrid_options o = options_or_default(options);
        *out = reinterpret_cast<hyt_hybrid *>(hybrid_create(csr, csc, o));
    });
}

int hyt_hybrid_destroy(hyt_hybrid *x) {
    return guarded([&] {
        if (!x) return;
        HybridImpl *h = reinterpret_cast<HybridImpl *>(x);
        cudaSetDevice(h->g.device);
        cudaStreamSynchronize(h->g.stream);
        cudaStreamSynchronize(h->copy);
        delete h;
    });
}

int hyt_hybrid_get_info(const hyt_hybrid *x, hyt_hybrid_info *out) {
    return guarded([&] {
        if (!x || !out) fail(HYT_E_INVALID, "NULL argument");
        const HybridImpl *h = reinterpret_cast<const HybridImpl *>(x);
        std::memset(out, 0, sizeof(*out));
        out->partitions = h->P;
        out->budget_bytes = h->budget;
        out->resident_bytes = h->resident_bytes;
        out->staging_bytes = 2 * h->stage_edges * (h->h_w && (h->flags & HYT_GRAPH_PUSH) ? 8 : 4) + h->cbytes;
        for (size_t p = 0; p < h->P; ++p) {
            if (!h->push_res.empty() && h->push_res[p]) ++out->resident_push_partitions;
            if (!h->pull_res.empty() && h->pull_res[p]) ++out->resident_pull_partitions;
        }
        out->h2d_gbs = h->link.h2d_gbs;
        out->zero_copy_gbs = h->link.zc_gbs;
        out->gather_gbs = h->link.gather_gbs;
        out->device_bytes = h->g.device_bytes() + h->push_res_cols.bytes() + h->push_res_w.bytes() +
                            h->pull_res_src.bytes() + h->stage_a[0].bytes() * 2 + h->stage_b[0].bytes() * 2 +
                            h->cdev.bytes();
    });
}

int hyt_hybrid_pagerank(hyt_hybrid *x, const hyt_pagerank_params *p, float *ranks_out, hyt_run_stats *stats,
                        hyt_hybrid_stats *tstats) {
    return guarded([&] {
        HybridImpl *h = impl(x);
        if (!p) fail(HYT_E_INVALID, "params is NULL");
        if (!(h->flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "hybrid graph was created without HYT_GRAPH_PULL");
        if (!(p->damping >= 0.0f && p->damping < 1.0f)) fail(HYT_E_INVALID, "PageRank damping_factor must be in [0, 1)");
        if (!(p->tolerance > 0.0f) || !std::isfinite(p->tolerance))
            fail(HYT_E_INVALID, "PageRank tolerance must be finite and positive");
        if (p->max_iterations == 0) fail(HYT_E_INVALID, "PageRank max_iterations must be greater than zero");
        HYT_CUDA(cudaSetDevice(h->g.device));
        h->stats = hyt_hybrid_stats{};
        HybridPull src(*h);
        hyt_run_stats st{};
        pagerank_partitioned(h->g, src, false, 0, p->damping, p->tolerance, p->max_iterations, h->g.stream, ranks_out,
                             &st);
        h->stats.device_ms = st.device_ms;
        h->stats.link_bytes = h->stats.filter_bytes + h->stats.compaction_bytes + h->stats.zero_copy_bytes;
        h->stats.link_gbs = h->stats.link_bytes / (st.device_ms * 1e-3) / 1e9;
        h->stats.h2d_peak_gbs = h->link.h2d_gbs;
        if (stats) *stats = st;
        if (tstats) *tstats = h->stats;
    });
}

int hyt_hybrid_sssp(hyt_hybrid *x, const hyt_sssp_params *p, uint32_t *dist_out, hyt_run_stats *stats,
                    hyt_hybrid_stats *tstats) {
    return guarded([&] {
        HybridImpl *h = impl(x);
        if (!p) fail(HYT_E_INVALID, "params is NULL");
        if (!(h->flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "hybrid graph was created without HYT_GRAPH_PUSH");
        HYT_CUDA(cudaSetDevice(h->g.device));
        h->stats = hyt_hybrid_stats{};
        HybridPush src(*h);
        hyt_run_stats st{};
        sssp_partitioned(h->g, src, p->source, p->max_rounds, h->g.stream, dist_out, &st);
        h->stats.device_ms = st.device_ms;
        h->stats.link_bytes = h->stats.filter_bytes + h->stats.compaction_bytes + h->stats.zero_copy_bytes;
        h->stats.link_gbs = h->stats.link_bytes / (st.device_ms * 1e-3) / 1e9;
        h->stats.h2d_peak_gbs = h->link.h2d_gbs;
        if (stats) *stats = st;
        if (tstats) *tstats = h->stats;
    });
}

}  // extern "C"
