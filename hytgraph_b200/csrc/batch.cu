// Multi-query engine and the batched-query C ABI (hyt_batch_*); the design
// is described in batch.cuh.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <tuple>
#include <mutex>
#include <map>
#include <string>

#include "batch.cuh"
#include "common.cuh"
#include "host_checks.hpp"
#include "graph.cuh"
#include "pagerank_core.cuh"
#include "sssp_core.cuh"

namespace hyt {
namespace {

using namespace ssc;
using prc::PRArgs;
using prc::PRBuffers;
using prc::PRHeader;
using prc::PRState;

enum : uint32_t { kFree = 0, kSSSP = 1, kPPR = 2 };

constexpr uint32_t kMaxSlots = 4096;
constexpr int kWorkThreads = 256;
constexpr size_t kSliceFloats = 2 * size_t(kTileCostMax) + 8;  // PPR tile staging per warp
constexpr int kSplitBlocks = 4;
constexpr int kInitBlocks = 64;
constexpr uint32_t kEndBlocks = 16;  // blocks per PPR slot in the end reduction
constexpr uint32_t kGrab = 4;        // units / hub tasks a warp takes at a time
constexpr bool kHotGlobal = true;    // hot sources read from the slot's hot_contrib array

struct Slot {
    uint32_t kind;        // kFree / kSSSP / kPPR
    uint32_t wk;          // SSSP weight kind
    uint32_t max_rounds;  // SSSP round cap
    uint32_t delta;       // SSSP bucket width (kNoDelta = one bucket)
};

// PPR per-query extras.  task_sums: (residual, dangling) of tile k at [k],
// of long row i at [num_tiles + i]; end blocks sum fixed stripes of it into
// block_sums, the last block sums those in index order.  hot_contrib[p]:
// the contributions of the graph's hot sources (tagged ids in in_sources)
// for iteration parity p, gathered once per iteration so that tasks read
// them with one load.
struct PRExtra {
    double2 *task_sums;
    double2 *block_sums;  // [kEndBlocks]
    uint32_t *end_ticket;
    float *hot_contrib[2];
    uint32_t num_tiles, num_long, num_chunks, num_hot;
};

struct SlotStatus {
    uint32_t done, iterations, converged, pad;
    double residual;
    unsigned long long edges, frontier;
};

}  // namespace

struct EngineArgs {
    Slot *slot;
    SSArgs *ss;
    PRArgs *pr;
    PRExtra *px;
    RoundView *rvs;       // per-slot round snapshot (SSSP), written by prep
    uint32_t n;           // slots [0, n) are examined
    uint32_t hub_degree;
    uint32_t *ss_base;    // [n + 1] SSSP unit prefix
    uint32_t *pr_base;    // [n + 1] PPR unit prefix
    uint4 *hubs;          // (slot, vertex, chunk, -)
    uint32_t hub_cap;
    uint32_t max_supersteps;
    // [0] hub tasks, [1] running after this superstep, [2] supersteps,
    // [3] overflow, [4] SSSP unit cursor, [5] hub cursor, [6] PPR unit cursor
    uint32_t *counters;
    cudaGraphConditionalHandle cond;
    uint32_t use_cond;
};

namespace {

__global__ void engine_init_kernel(const EngineArgs *__restrict__ eap, uint32_t s0) {
    const EngineArgs ea = *eap;
    const uint32_t q = s0 + blockIdx.y;
    const Slot sl = ea.slot[q];
    const uint32_t stride = gridDim.x * blockDim.x;
    if (sl.kind == kSSSP) {
        const SSArgs a = ea.ss[q];
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.V; v += stride) init_vertex(a, v);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.queue[0][0] = a.source;
            SSHeader *h = a.hdr;
            h->qsize[0] = 1;
            h->max_rounds = sl.max_rounds;
            h->delta = sl.delta;
            h->threshold = (sl.wk == HYT_WEIGHTS_F32 || sl.delta == kNoDelta) ? 0xFFFFFFFFu : sl.delta;
        }
    } else if (sl.kind == kPPR) {
        // x_0 = e_s (the state block arrives zeroed)
        const PRArgs a = ea.pr[q];
        const PRExtra x = ea.px[q];
        const uint32_t s = a.source;
        const uint32_t od = a.out_deg[s];
        const float c0 = od ? __fdiv_rn(1.0f, static_cast<float>(od)) : 0.0f;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.rank[0][s] = 1.0f;
            a.contrib[0][s] = c0;
            a.dangling[0] = od ? 0.0 : 1.0;
        }
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < x.num_hot; i += stride)
            if (a.hot_vertex[i] == s) x.hot_contrib[0][i] = c0;
    }
}

__global__ void engine_split_kernel(const EngineArgs *__restrict__ eap) {
    const EngineArgs ea = *eap;
    const uint32_t q = blockIdx.y;
    if (q >= ea.n || ea.slot[q].kind != kSSSP) return;
    const SSArgs a = ea.ss[q];
    const SSHeader *h = a.hdr;
    if (*(volatile const uint32_t *)&h->done || !*(volatile const uint32_t *)&h->pending) return;
    const uint32_t n = (h->phase & 1) ? h->fsize[1] : h->fsize[0];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) split_entry(a, i);
}

// Work units of slot q this superstep (SSSP: 32-vertex frontier blocks,
// PPR: chunk tasks + tiles); snapshots the SSSP round view.
__device__ __forceinline__ void slot_units(const EngineArgs &ea, uint32_t q, uint32_t &ss, uint32_t &pr,
                                           bool snapshot) {
    ss = pr = 0;
    const Slot sl = ea.slot[q];
    if (sl.kind == kSSSP) {
        const SSArgs a = ea.ss[q];
        if (*(volatile const uint32_t *)&a.hdr->done) return;
        const RoundView rv = round_view(a);
        if (snapshot) ea.rvs[q] = rv;
        ss = (rv.qn + 31) / 32;
    } else if (sl.kind == kPPR) {
        if (*(volatile const uint32_t *)&ea.pr[q].hdr->done) return;
        const PRExtra x = ea.px[q];
        pr = x.num_chunks + x.num_tiles;
    }
}

// Block-wide exclusive scan of one value per thread (1024 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s_warp, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __syncthreads();
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = (lane < static_cast<int>(blockDim.x >> 5)) ? s_warp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        s_warp[lane] = wi - w;
        if (lane == 31) s_warp[32] = wi;
    }
    __syncthreads();
    total = s_warp[32];
    return s_warp[warp] + incl - v;
}

// One CTA of 1024 threads: per-slot SSSP and PPR unit prefixes, SSSP round
// snapshots, cursors reset.
__global__ void __launch_bounds__(1024) engine_prep_kernel(const EngineArgs *__restrict__ eap) {
    __shared__ uint32_t s_warp[33];
    const EngineArgs ea = *eap;
    const uint32_t n = ea.n;
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(n, b + per);
    uint32_t ss_sum = 0, pr_sum = 0;
    for (uint32_t q = b; q < e; ++q) {
        uint32_t s, p;
        slot_units(ea, q, s, p, true);
        ss_sum += s;
        pr_sum += p;
    }
    uint32_t ss_total, pr_total;
    uint32_t ss_at = block_exclusive_scan(ss_sum, s_warp, ss_total);
    uint32_t pr_at = block_exclusive_scan(pr_sum, s_warp, pr_total);
    for (uint32_t q = b; q < e; ++q) {
        ea.ss_base[q] = ss_at;
        ea.pr_base[q] = pr_at;
        uint32_t s, p;
        slot_units(ea, q, s, p, false);
        ss_at += s;
        pr_at += p;
    }
    if (threadIdx.x == 0) {
        ea.ss_base[n] = ss_total;
        ea.pr_base[n] = pr_total;
        ea.counters[0] = 0;
        ea.counters[4] = 0;
        ea.counters[5] = 0;
        ea.counters[6] = 0;
    }
}

// Slot of unit u: the last q with base[q] <= u (base in shared memory).
__device__ __forceinline__ uint32_t find_slot(const uint32_t *base, uint32_t n, uint32_t u) {
    uint32_t lo = 0, hi = n;  // base[lo] <= u < base[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (base[mid] <= u) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Next kGrab-sized range of a global cursor for this warp (lane 0 takes it).
__device__ __forceinline__ uint32_t grab(uint32_t *cursor, int lane) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(cursor, kGrab);
    return __shfl_sync(0xffffffffu, c, 0);
}

// Adds the warp's relaxation count to the slot's header; all 32 lanes.
__device__ __forceinline__ void flush_relaxed(const SSArgs &a, unsigned long long &relaxed, int lane) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) relaxed += __shfl_xor_sync(0xffffffffu, relaxed, o);
    if (lane == 0 && relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
    relaxed = 0;
}

// SSSP frontier blocks of every SSSP slot.  Warps take kGrab consecutive
// units at a time; a slot's arguments are reloaded only when the slot
// changes.
__global__ void __launch_bounds__(kWorkThreads, 3) engine_sssp_kernel(const EngineArgs *__restrict__ eap) {
    extern __shared__ __align__(16) uint32_t s_base[];
    const EngineArgs ea = *eap;
    const uint32_t n = ea.n;
    for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) s_base[i] = ea.ss_base[i];
    __syncthreads();
    const uint32_t total = s_base[n];
    const int lane = threadIdx.x & 31;
    uint32_t cq = ~0u, wk = 0;
    SSArgs a{};
    RoundView rv{};
    unsigned long long relaxed = 0, improved = 0;
    uint32_t *hub_count = ea.counters + 0;
    for (uint32_t c = grab(ea.counters + 4, lane); c < total; c = grab(ea.counters + 4, lane)) {
        const uint32_t end = min(total, c + kGrab);
        for (uint32_t u = c; u < end; ++u) {
            const uint32_t q = find_slot(s_base, n, u);
            if (q != cq) {  // warp-uniform
                if (cq != ~0u) flush_relaxed(a, relaxed, lane);
                a = ea.ss[q];
                rv = ea.rvs[q];
                wk = ea.slot[q].wk;
                cq = q;
            }
            auto hub = [&](uint32_t v, uint32_t nch) {
                const uint32_t base = atomicAdd(hub_count, nch);
                if (base + nch > ea.hub_cap) {  // cannot happen within the admitted bound; reported, never written
                    atomicExch(&ea.counters[3], 1u);
                    return;
                }
                for (uint32_t k = 0; k < nch; ++k) ea.hubs[base + k] = make_uint4(q, v, k, 0u);
            };
            const uint32_t i0 = (u - s_base[q]) * 32;
            if (wk == HYT_WEIGHTS_U32) {
                expand_warp<HYT_WEIGHTS_U32, false>(a, rv, i0, lane, ea.hub_degree, relaxed, improved, hub);
            } else if (wk == HYT_WEIGHTS_NONE) {
                expand_warp<HYT_WEIGHTS_NONE, false>(a, rv, i0, lane, ea.hub_degree, relaxed, improved, hub);
            } else {
                expand_warp<HYT_WEIGHTS_F32, false>(a, rv, i0, lane, ea.hub_degree, relaxed, improved, hub);
            }
        }
    }
    if (cq != ~0u) flush_relaxed(a, relaxed, lane);
}

// PPR tasks of every PPR slot: warps take units round-robin (every task
// costs at most one long-row chunk; at any moment the grid works inside
// one slot's unit range, so its contributions stay in L2); a slot's
// arguments are read per unit (L1-resident); hot sources come from the
// slot's hot_contrib array.
__global__ void __launch_bounds__(kWorkThreads) engine_ppr_kernel(const EngineArgs *__restrict__ eap) {
    extern __shared__ __align__(16) float s_dyn[];
    const EngineArgs ea = *eap;
    const uint32_t n = ea.n;
    uint32_t *s_base = reinterpret_cast<uint32_t *>(s_dyn + (kWorkThreads / 32) * kSliceFloats);
    for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) s_base[i] = ea.pr_base[i];
    __syncthreads();
    const uint32_t total = s_base[n];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *sv = s_dyn + warp * kSliceFloats;
    const uint64_t pol = dev::policy_evict_last();
    const uint32_t nwarps = gridDim.x * (kWorkThreads / 32);
    for (uint32_t u = blockIdx.x * (kWorkThreads / 32) + warp; u < total; u += nwarps) {
        const uint32_t q = find_slot(s_base, n, u);
        const uint32_t t = u - s_base[q];
        const PRArgs a = ea.pr[q];
        const PRExtra x = ea.px[q];
        const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
        const PRBuffers b = prc::buffers(a, it);
        const PRState ps = prc::make_state(a, a.dangling[it]);
        const float *hot = x.hot_contrib[it & 1];
        double res = 0.0, dang = 0.0;
        if (t < x.num_chunks) {
            const uint32_t li = prc::chunk_task<kHotGlobal>(a, ps, b, a.in_src, hot, t, pol, lane, res, dang);
            if (li != ~0u && lane == 0) x.task_sums[x.num_tiles + li] = make_double2(res, dang);
        } else {
            const uint64_t k = t - x.num_chunks;
            prc::tile_task<kHotGlobal>(a, ps, b, a.in_src, hot, sv, k, pol, lane, res, dang);
            res = dev::warp_sum(res);
            dang = dev::warp_sum(dang);
            if (lane == 0) x.task_sums[k] = make_double2(res, dang);
        }
    }
}

__global__ void __launch_bounds__(kWorkThreads, 3) engine_hub_kernel(const EngineArgs *__restrict__ eap) {
    const EngineArgs ea = *eap;
    const uint32_t n = min(*(volatile uint32_t *)&ea.counters[0], ea.hub_cap);
    const int lane = threadIdx.x & 31;
    uint32_t cq = ~0u, wk = 0;
    SSArgs a{};
    RoundView rv{};
    unsigned long long improved = 0;
    for (uint32_t c = grab(ea.counters + 5, lane); c < n; c = grab(ea.counters + 5, lane)) {
        const uint32_t end = min(n, c + kGrab);
        for (uint32_t t = c; t < end; ++t) {
            const uint4 h = ea.hubs[t];
            if (h.x != cq) {
                a = ea.ss[h.x];
                rv = ea.rvs[h.x];
                wk = ea.slot[h.x].wk;
                cq = h.x;
            }
            if (wk == HYT_WEIGHTS_U32) {
                hub_chunk<HYT_WEIGHTS_U32>(a, rv, a.cols, a.weights, h.y, h.z, lane, improved);
            } else if (wk == HYT_WEIGHTS_NONE) {
                hub_chunk<HYT_WEIGHTS_NONE>(a, rv, a.cols, a.weights, h.y, h.z, lane, improved);
            } else {
                hub_chunk<HYT_WEIGHTS_F32>(a, rv, a.cols, a.weights, h.y, h.z, lane, improved);
            }
        }
    }
}

// Grid (kEndBlocks, slots).  SSSP: block 0 closes the round.  PPR: block b
// sums stripe b of the task partials and gathers stripe b of the next
// iteration's hot contributions; the last block to arrive sums the
// kEndBlocks stripe sums in index order (a fixed association, independent
// of the other slots) and applies the stop rule.
__global__ void engine_end_kernel(const EngineArgs *__restrict__ eap) {
    __shared__ double s_red[32];
    __shared__ uint32_t s_last;
    const EngineArgs ea = *eap;
    const uint32_t q = blockIdx.y;
    if (q >= ea.n) return;
    const Slot sl = ea.slot[q];
    if (sl.kind == kSSSP) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            SSHeader *h = ea.ss[q].hdr;
            if (!h->done && !round_end(h)) atomicAdd(&ea.counters[1], 1u);
        }
        return;
    }
    if (sl.kind != kPPR) return;
    const PRArgs a = ea.pr[q];
    if (*(volatile uint32_t *)&a.hdr->done) return;
    const PRExtra x = ea.px[q];
    const uint32_t it = a.hdr->iter;
    const uint32_t m = x.num_tiles + x.num_long;
    const uint32_t stripe = (m + kEndBlocks - 1) / kEndBlocks;
    const uint32_t lo = min(m, blockIdx.x * stripe), hi = min(m, lo + stripe);
    double r = 0.0, d = 0.0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double2 v = x.task_sums[i];
        r += v.x;
        d += v.y;
    }
    r = dev::block_sum(r, s_red);
    __syncthreads();
    d = dev::block_sum(d, s_red);
    // hot contributions of the next iteration (its contributions are final now)
    const float *cnxt = ((it + 1) & 1) ? a.contrib[1] : a.contrib[0];
    float *hnxt = x.hot_contrib[(it + 1) & 1];
    const uint32_t hs = (x.num_hot + kEndBlocks - 1) / kEndBlocks;
    for (uint32_t i = blockIdx.x * hs + threadIdx.x; i < min(x.num_hot, (blockIdx.x + 1) * hs); i += blockDim.x)
        hnxt[i] = cnxt[a.hot_vertex[i]];
    if (threadIdx.x == 0) {
        x.block_sums[blockIdx.x] = make_double2(r, d);
        __threadfence();
        const uint32_t t = atomicAdd(x.end_ticket, 1u) + 1u;
        s_last = (t % kEndBlocks == 0) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    double rs = 0.0, ds = 0.0;
    for (uint32_t k = 0; k < kEndBlocks; ++k) {
        const double2 v = __ldcg(x.block_sums + k);
        rs += v.x;
        ds += v.y;
    }
    a.residual[it] = rs;
    a.dangling[it + 1] = ds;
    prc::end_iteration(a, it);
    if (!a.hdr->done) atomicAdd(&ea.counters[1], 1u);
}

__global__ void engine_cond_kernel(const EngineArgs *__restrict__ eap) {
    const EngineArgs ea = *eap;
    const uint32_t running = ea.counters[1];
    ea.counters[1] = 0;
    const uint32_t steps = ++ea.counters[2];
    if (ea.use_cond && (running == 0 || steps >= ea.max_supersteps || ea.counters[3]))
        cudaGraphSetConditional(ea.cond, 0);
}

__global__ void engine_status_kernel(const EngineArgs *__restrict__ eap, SlotStatus *out) {
    const EngineArgs ea = *eap;
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ea.n) return;
    const Slot sl = ea.slot[q];
    SlotStatus st{};
    if (sl.kind == kSSSP) {
        const SSHeader *h = ea.ss[q].hdr;
        st.done = h->done;
        st.iterations = h->round;
        st.converged = h->converged;
        st.edges = h->relaxations;
        st.frontier = h->frontier_total;
    } else if (sl.kind == kPPR) {
        const PRHeader *h = ea.pr[q].hdr;
        st.done = h->done;
        st.iterations = h->iter;
        st.converged = h->converged;
        st.residual = h->last_residual;
    }
    out[q] = st;
}

uint64_t align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

int ppr_kernel_smem(uint32_t cap) {
    return static_cast<int>((kWorkThreads / 32) * kSliceFloats * sizeof(float) + (cap + 1) * sizeof(uint32_t));
}

int sssp_kernel_smem(uint32_t cap) { return static_cast<int>((cap + 1) * sizeof(uint32_t)); }

}  // namespace

// ------------------------------------------------------------------ host --
struct EngineHost {
    EngineArgs args{};  // last uploaded
    std::vector<Slot> slot;
    std::vector<SSArgs> ss;
    std::vector<PRArgs> pr;
    std::vector<PRExtra> px;
    DeviceArray<Slot> d_slot;
    DeviceArray<SSArgs> d_ss;
    DeviceArray<PRArgs> d_pr;
    DeviceArray<PRExtra> d_px;
    DeviceArray<RoundView> d_rvs;
    DeviceArray<SlotStatus> d_status;
    PinnedArray<SlotStatus> h_status;
};

QueryEngine::QueryEngine(int device, cudaStream_t stream, uint64_t budget_bytes)
    : device_(device), stream_(stream), budget_(budget_bytes), host_(std::make_unique<EngineHost>()) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    HYT_CUDA(cudaMemPoolCreate(&pool_, &props));
    uint64_t keep = std::numeric_limits<uint64_t>::max();
    HYT_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
    counters_.allocate(8);
    HYT_CUDA(cudaMemsetAsync(counters_.get(), 0, 32, stream_));
    d_args_.allocate(1);
    grow(64);
}

QueryEngine::~QueryEngine() {
    cudaStreamSynchronize(stream_);
    for (auto &s : slots_)
        if (s.mem) cudaFreeAsync(s.mem, stream_);
    cudaStreamSynchronize(stream_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (step_exec_) cudaGraphExecDestroy(step_exec_);
    if (step_graph_) cudaGraphDestroy(step_graph_);
    if (pool_) cudaMemPoolDestroy(pool_);
}

void QueryEngine::set_graphs(const std::vector<GraphImpl *> &graphs) { graphs_ = graphs; }

void QueryEngine::grow(uint32_t cap) {
    if (cap <= cap_) return;
    cap = std::min(cap, kMaxSlots);
    EngineHost &h = *host_;
    HYT_CUDA(cudaStreamSynchronize(stream_));
    h.slot.resize(cap, Slot{kFree, 0, 0, 0});
    h.ss.resize(cap, SSArgs{});
    h.pr.resize(cap, PRArgs{});
    h.px.resize(cap, PRExtra{});
    h.d_slot.allocate(cap);
    h.d_ss.allocate(cap);
    h.d_pr.allocate(cap);
    h.d_px.allocate(cap);
    h.d_rvs.allocate(cap);
    h.d_status.allocate(cap);
    h.h_status.allocate(cap);
    HYT_CUDA(cudaMemcpyAsync(h.d_slot.get(), h.slot.data(), cap * sizeof(Slot), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_ss.get(), h.ss.data(), cap * sizeof(SSArgs), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_pr.get(), h.pr.data(), cap * sizeof(PRArgs), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_px.get(), h.px.data(), cap * sizeof(PRExtra), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaStreamSynchronize(stream_));
    unit_base_.allocate(2 * (cap + 1));  // SSSP prefix, then PPR prefix
    slots_.resize(cap);
    cap_ = cap;
    HYT_CUDA(cudaFuncSetAttribute(engine_ppr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  ppr_kernel_smem(kMaxSlots)));
    // the cached graphs' grid sizes depend on the capacity
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (step_exec_) cudaGraphExecDestroy(step_exec_);
    if (step_graph_) cudaGraphDestroy(step_graph_);
    exec_ = step_exec_ = nullptr;
    graph_ = step_graph_ = nullptr;
    args_dirty_ = true;
}

void QueryEngine::validate(const hyt_query &q) const {
    if (q.graph >= graphs_.size()) fail(HYT_E_INVALID, "query graph index is out of range");
    const GraphImpl &g = *graphs_[q.graph];
    if (q.kind == HYT_QUERY_SSSP) {
        if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "SSSP queries need graphs built with HYT_GRAPH_PUSH");
        if (q.source >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
        if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
    } else if (q.kind == HYT_QUERY_PPR) {
        if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "PPR queries need graphs built with HYT_GRAPH_PULL");
        if (q.source >= g.V) fail(HYT_E_INVALID, "personalized PageRank source vertex is out of range");
        if (!(q.restart >= 0.0f && q.restart <= 1.0f))
            fail(HYT_E_INVALID, "personalized PageRank restart must be in (0, 1]");
        if (!(q.tolerance >= 0.0f) || !std::isfinite(q.tolerance))
            fail(HYT_E_INVALID, "personalized PageRank tolerance must be finite and positive");
    } else {
        fail(HYT_E_INVALID, "unknown query kind");
    }
}

namespace {
uint32_t ppr_iters(const hyt_query &q) { return q.max_iterations ? q.max_iterations : 100u; }

uint64_t sssp_round_cap(const hyt_query &q, const GraphImpl &g) {
    return q.max_iterations ? q.max_iterations : std::min<uint64_t>(4 * g.V + 1024, 0x7FFFFFFFull);
}
}  // namespace

uint64_t QueryEngine::state_bytes(const hyt_query &q) const {
    const GraphImpl &g = *graphs_[q.graph];
    const uint64_t V = g.V;
    if (q.kind == HYT_QUERY_SSSP) return align256(sizeof(SSHeader)) + 7 * align256(V * 4 + 16);
    const uint64_t it = ppr_iters(q);
    return align256(sizeof(PRHeader)) + 4 * align256(V * 4 + 16) + align256(g.num_chunks * 8 + 16) +
           align256(g.num_long * 4 + 16) + align256((g.num_tiles + g.num_long) * 16 + 16) + 2 * align256((it + 2) * 8) +
           align256(kEndBlocks * 16) + align256(16) + 2 * align256(uint64_t(g.num_hot) * 4 + 16);
}

int QueryEngine::admit(const hyt_query &q, uint64_t tag) {
    const uint64_t need = state_bytes(q);
    if (in_use_ + need > budget_) return -1;
    int s = -1;
    for (uint32_t i = 0; i < cap_; ++i)
        if (!slots_[i].used) {
            s = static_cast<int>(i);
            break;
        }
    if (s < 0) {
        if (cap_ >= kMaxSlots) return -1;
        const uint32_t old = cap_;
        grow(cap_ * 2);
        s = static_cast<int>(old);
    }
    const GraphImpl &g = *graphs_[q.graph];
    void *mem = nullptr;
    HYT_CUDA(cudaMallocFromPoolAsync(&mem, need, pool_, stream_));
    HYT_CUDA(cudaMemsetAsync(mem, 0, need, stream_));
    unsigned char *p = static_cast<unsigned char *>(mem);
    auto take = [&](uint64_t bytes) {
        unsigned char *r = p;
        p += align256(bytes);
        return r;
    };
    EngineHost &h = *host_;
    const uint64_t V = g.V;
    Slot sl{};
    if (q.kind == HYT_QUERY_SSSP) {
        SSArgs a{};
        a.hdr = reinterpret_cast<SSHeader *>(take(sizeof(SSHeader)));
        a.row_off = g.row_offsets.get();
        a.cols = g.cols.get();
        a.weights = g.weights.get();
        a.dist = reinterpret_cast<uint32_t *>(take(V * 4 + 16));
        a.stamp = reinterpret_cast<uint32_t *>(take(V * 4 + 16));
        a.fstamp = reinterpret_cast<uint32_t *>(take(V * 4 + 16));
        for (int i = 0; i < 2; ++i) {
            a.queue[i] = reinterpret_cast<uint32_t *>(take(V * 4 + 16));
            a.far[i] = reinterpret_cast<uint32_t *>(take(V * 4 + 16));
        }
        a.V = static_cast<uint32_t>(V);
        a.source = graph_vertex(g, q.source, stream_);  // internal id on hub-ordered graphs
        a.inf = (g.weight_kind == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
        h.ss[s] = a;
        sl.kind = kSSSP;
        sl.wk = g.weight_kind;
        sl.max_rounds = static_cast<uint32_t>(sssp_round_cap(q, g));
        const uint32_t mean = std::max<uint32_t>(1, g.default_delta / 2);
        sl.delta = (tuning_.delta_mult == 0 || g.weight_kind == HYT_WEIGHTS_F32)
                       ? kNoDelta
                       : static_cast<uint32_t>(std::min<uint64_t>(uint64_t(tuning_.delta_mult) * mean, 0xFFFFFFFEull));
        slots_[s].hub = g.E / kHubChunk + g.E / std::max<uint32_t>(tuning_.hub_degree, 1) + 2;
        hub_need_ += slots_[s].hub;
    } else {
        PRArgs a{};
        const uint32_t it = ppr_iters(q);
        const float restart = q.restart > 0.0f ? q.restart : 0.15f;
        a.hdr = reinterpret_cast<PRHeader *>(take(sizeof(PRHeader)));
        a.in_off = g.in_offsets.get();
        a.in_src = g.in_sources.get();
        a.out_deg = g.out_degree.get();
        a.tile_start = g.tile_start.get();
        a.long_rows = g.long_rows.get();
        a.chunk_tasks = g.chunk_tasks.get();
        a.hot_vertex = g.hot_vertex.get();
        a.num_hot = g.num_hot;
        a.tile_cost = g.tile_cost;
        for (int i = 0; i < 2; ++i) a.rank[i] = reinterpret_cast<float *>(take(V * 4 + 16));
        for (int i = 0; i < 2; ++i) a.contrib[i] = reinterpret_cast<float *>(take(V * 4 + 16));
        a.partial = reinterpret_cast<float2 *>(take(g.num_chunks * 8 + 16));
        a.ticket = reinterpret_cast<uint32_t *>(take(g.num_long * 4 + 16));
        PRExtra x{};
        x.task_sums = reinterpret_cast<double2 *>(take((g.num_tiles + g.num_long) * 16 + 16));
        x.num_tiles = static_cast<uint32_t>(g.num_tiles);
        x.num_long = static_cast<uint32_t>(g.num_long);
        x.num_chunks = static_cast<uint32_t>(g.num_chunks);
        x.num_hot = g.num_hot;
        a.residual = reinterpret_cast<double *>(take((it + 2) * 8));
        a.dangling = reinterpret_cast<double *>(take((it + 2) * 8));
        x.block_sums = reinterpret_cast<double2 *>(take(kEndBlocks * 16));
        x.end_ticket = reinterpret_cast<uint32_t *>(take(16));
        for (int i = 0; i < 2; ++i) x.hot_contrib[i] = reinterpret_cast<float *>(take(uint64_t(g.num_hot) * 4 + 16));
        a.num_tiles = g.num_tiles;
        a.num_chunks = static_cast<uint32_t>(g.num_chunks);
        a.V = static_cast<uint32_t>(V);
        a.damping = 1.0f - restart;
        a.base = 0.0f;
        a.tolerance = q.tolerance > 0.0f ? q.tolerance : 1e-6f;
        a.max_iter = it;
        a.source = graph_vertex(g, q.source, stream_);
        a.personalized = 1;
        a.use_cond = 0;
        h.pr[s] = a;
        h.px[s] = x;
        sl.kind = kPPR;
    }
    h.slot[s] = sl;
    // pageable sources: the copies are staged before the calls return
    HYT_CUDA(cudaMemcpyAsync(h.d_slot.get() + s, &h.slot[s], sizeof(Slot), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_ss.get() + s, &h.ss[s], sizeof(SSArgs), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_pr.get() + s, &h.pr[s], sizeof(PRArgs), cudaMemcpyHostToDevice, stream_));
    HYT_CUDA(cudaMemcpyAsync(h.d_px.get() + s, &h.px[s], sizeof(PRExtra), cudaMemcpyHostToDevice, stream_));
    SlotHost &sh = slots_[s];
    if (q.kind != HYT_QUERY_SSSP) sh.hub = 0;
    sh.used = sh.running = true;
    sh.q = q;
    sh.tag = tag;
    sh.bytes = need;
    sh.mem = mem;
    in_use_ += need;
    ++used_slots_;
    ++running_;
    hi_ = std::max<uint32_t>(hi_, static_cast<uint32_t>(s) + 1);
    ensure_hub_capacity();
    upload_args(false);
    const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((V + 255) / 256, kInitBlocks));
    engine_init_kernel<<<dim3(std::max(blocks, 1u), 1), 256, 0, stream_>>>(d_args_.get(), static_cast<uint32_t>(s));
    HYT_CUDA(cudaGetLastError());
    ++launches_;
    return s;
}

void QueryEngine::ensure_hub_capacity() {
    if (hubs_.count >= hub_need_) return;
    HYT_CUDA(cudaStreamSynchronize(stream_));
    hubs_.allocate(std::max<uint64_t>(hub_need_, hubs_.count * 2));
    args_dirty_ = true;
}

namespace {
int occupancy(const void *f, int smem) {
    int per_sm = 0;
    HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kWorkThreads, smem));
    return std::max(per_sm, 1);
}
}  // namespace

int QueryEngine::ppr_grid() const {
    static int per_sm = 0;
    if (per_sm == 0) per_sm = occupancy(reinterpret_cast<const void *>(engine_ppr_kernel), ppr_kernel_smem(kMaxSlots));
    return sm_count() * per_sm;
}

int QueryEngine::work_grid() const {
    static int per_sm = 0;
    if (per_sm == 0)
        per_sm = occupancy(reinterpret_cast<const void *>(engine_sssp_kernel), sssp_kernel_smem(kMaxSlots));
    const int c = tuning_.ctas_per_sm ? std::min<int>(static_cast<int>(tuning_.ctas_per_sm), per_sm) : per_sm;
    return sm_count() * c;
}

void QueryEngine::upload_args(bool use_cond) {
    EngineHost &h = *host_;
    EngineArgs a{};
    a.slot = h.d_slot.get();
    a.ss = h.d_ss.get();
    a.pr = h.d_pr.get();
    a.px = h.d_px.get();
    a.rvs = h.d_rvs.get();
    a.n = hi_;
    a.hub_degree = std::max<uint32_t>(tuning_.hub_degree, 1);
    a.ss_base = unit_base_.get();
    a.pr_base = unit_base_.get() + cap_ + 1;
    a.hubs = hubs_.get();
    a.hub_cap = static_cast<uint32_t>(std::min<uint64_t>(hubs_.count, 0xFFFFFFFFull));
    a.max_supersteps = max_supersteps_;
    a.counters = counters_.get();
    a.cond = use_cond ? cond_ : cudaGraphConditionalHandle{};
    a.use_cond = use_cond ? 1u : 0u;
    if (!args_dirty_ && std::memcmp(&a, &h.args, sizeof(a)) == 0) return;
    h.args = a;
    HYT_CUDA(cudaMemcpyAsync(d_args_.get(), &h.args, sizeof(a), cudaMemcpyHostToDevice, stream_));
    args_dirty_ = false;
}

void QueryEngine::launch_superstep_kernels(cudaStream_t s) {
    const int grid = work_grid();
    const EngineArgs *d = d_args_.get();
    engine_split_kernel<<<dim3(kSplitBlocks, cap_), 256, 0, s>>>(d);
    engine_prep_kernel<<<1, 1024, 0, s>>>(d);
    engine_sssp_kernel<<<grid, kWorkThreads, sssp_kernel_smem(cap_), s>>>(d);
    engine_ppr_kernel<<<ppr_grid(), kWorkThreads, ppr_kernel_smem(cap_), s>>>(d);
    engine_hub_kernel<<<grid, kWorkThreads, 0, s>>>(d);
    engine_end_kernel<<<dim3(kEndBlocks, cap_), 256, 0, s>>>(d);
    engine_cond_kernel<<<1, 1, 0, s>>>(d);
    HYT_CUDA(cudaGetLastError());
}

void QueryEngine::add_superstep_nodes(cudaGraph_t body, int grid) {
    EngineArgs *d = d_args_.get();
    void *kargs[] = {&d};
    struct K {
        void *f;
        dim3 grid, block;
        unsigned smem;
    };
    const K ks[] = {
        {reinterpret_cast<void *>(engine_split_kernel), dim3(kSplitBlocks, cap_), dim3(256), 0u},
        {reinterpret_cast<void *>(engine_prep_kernel), dim3(1), dim3(1024), 0u},
        {reinterpret_cast<void *>(engine_sssp_kernel), dim3(grid), dim3(kWorkThreads),
         static_cast<unsigned>(sssp_kernel_smem(cap_))},
        {reinterpret_cast<void *>(engine_ppr_kernel), dim3(ppr_grid()), dim3(kWorkThreads),
         static_cast<unsigned>(ppr_kernel_smem(cap_))},
        {reinterpret_cast<void *>(engine_hub_kernel), dim3(grid), dim3(kWorkThreads), 0u},
        {reinterpret_cast<void *>(engine_end_kernel), dim3(kEndBlocks, cap_), dim3(256), 0u},
        {reinterpret_cast<void *>(engine_cond_kernel), dim3(1), dim3(1), 0u},
    };
    cudaGraphNode_t prev = nullptr;
    for (const K &k : ks) {
        cudaKernelNodeParams kp = {};
        kp.func = k.f;
        kp.gridDim = k.grid;
        kp.blockDim = k.block;
        kp.sharedMemBytes = k.smem;
        kp.kernelParams = kargs;
        cudaGraphNode_t node;
        HYT_CUDA(cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
        prev = node;
    }
}

void QueryEngine::build_step_exec() {
    const int grid = work_grid();
    if (step_exec_ && step_grid_ == grid) return;
    if (step_exec_) cudaGraphExecDestroy(step_exec_);
    if (step_graph_) cudaGraphDestroy(step_graph_);
    step_exec_ = nullptr;
    HYT_CUDA(cudaGraphCreate(&step_graph_, 0));
    add_superstep_nodes(step_graph_, grid);
    HYT_CUDA(cudaGraphInstantiate(&step_exec_, step_graph_, 0));
    step_grid_ = grid;
}

void QueryEngine::step() {
    if (running_ == 0) return;
    build_step_exec();
    max_supersteps_ = 0x7FFFFFFF;
    upload_args(false);
    HYT_CUDA(cudaGraphLaunch(step_exec_, stream_));
    ++launches_;
}

void QueryEngine::build_graph_exec() {
    const int grid = work_grid();
    if (exec_ && exec_grid_ == grid) return;
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    HYT_CUDA(cudaGraphCreate(&graph_, 0));
    HYT_CUDA(cudaGraphConditionalHandleCreate(&cond_, graph_, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond_;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    HYT_CUDA(cudaGraphAddNode(&cnode, graph_, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    add_superstep_nodes(body, grid);
    HYT_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    exec_grid_ = grid;
    args_dirty_ = true;
}

uint32_t QueryEngine::run_to_completion(bool use_graph) {
    if (running_ == 0) return 0;
    // superstep cap: the longest admitted query's own cap, plus one
    uint64_t cap = 1;
    for (uint32_t i = 0; i < hi_; ++i) {
        const SlotHost &sh = slots_[i];
        if (!sh.running) continue;
        const GraphImpl &g = *graphs_[sh.q.graph];
        const uint64_t c = sh.q.kind == HYT_QUERY_SSSP ? sssp_round_cap(sh.q, g) : ppr_iters(sh.q);
        cap = std::max(cap, c + 1);
    }
    max_supersteps_ = static_cast<uint32_t>(std::min<uint64_t>(cap, 0x7FFFFFFFull));
    HYT_CUDA(cudaMemsetAsync(counters_.get(), 0, 32, stream_));
    uint32_t steps = 0;
    EngineHost &h = *host_;
    if (use_graph) {
        build_graph_exec();
        upload_args(true);
        HYT_CUDA(cudaGraphLaunch(exec_, stream_));
        launches_ += 1;
        uint32_t c[4] = {0, 0, 0, 0};
        HYT_CUDA(cudaMemcpyAsync(c, counters_.get(), 16, cudaMemcpyDeviceToHost, stream_));
        HYT_CUDA(cudaStreamSynchronize(stream_));
        steps = c[2];
        if (c[3]) fail(HYT_E_INTERNAL, "batch hub task list overflowed");
    } else {
        upload_args(false);
        for (;;) {
            launch_superstep_kernels(stream_);
            launches_ += 7;
            engine_status_kernel<<<(hi_ + 255) / 256, 256, 0, stream_>>>(d_args_.get(), h.d_status.get());
            uint32_t c[4] = {0, 0, 0, 0};
            HYT_CUDA(cudaMemcpyAsync(c, counters_.get(), 16, cudaMemcpyDeviceToHost, stream_));
            HYT_CUDA(cudaMemcpyAsync(h.h_status.ptr, h.d_status.get(), hi_ * sizeof(SlotStatus),
                                     cudaMemcpyDeviceToHost, stream_));
            HYT_CUDA(cudaStreamSynchronize(stream_));
            steps = c[2];
            if (c[3]) fail(HYT_E_INTERNAL, "batch hub task list overflowed");
            bool any = false;
            for (uint32_t i = 0; i < hi_; ++i)
                if (slots_[i].running && !h.h_status.ptr[i].done) any = true;
            if (!any || steps >= max_supersteps_) break;
        }
    }
    return steps;
}

void QueryEngine::run_supersteps(uint32_t n) {
    if (running_ == 0) return;
    max_supersteps_ = 0x7FFFFFFF;
    upload_args(false);
    for (uint32_t i = 0; i < n; ++i) launch_superstep_kernels(stream_);
    launches_ += 7ull * n;
}

std::vector<std::pair<int, uint64_t>> QueryEngine::finished() {
    std::vector<std::pair<int, uint64_t>> out;
    if (hi_ == 0) return out;
    EngineHost &h = *host_;
    engine_status_kernel<<<(hi_ + 255) / 256, 256, 0, stream_>>>(d_args_.get(), h.d_status.get());
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaMemcpyAsync(h.h_status.ptr, h.d_status.get(), hi_ * sizeof(SlotStatus), cudaMemcpyDeviceToHost,
                             stream_));
    HYT_CUDA(cudaStreamSynchronize(stream_));
    for (uint32_t i = 0; i < hi_; ++i) {
        SlotHost &sh = slots_[i];
        if (sh.used && sh.running && h.h_status.ptr[i].done) {
            sh.running = false;
            --running_;
            out.emplace_back(static_cast<int>(i), sh.tag);
        }
    }
    return out;
}

void QueryEngine::retire(int s, hyt_query_result *res) {
    SlotHost &sh = slots_[s];
    if (!sh.used) fail(HYT_E_INTERNAL, "retiring a free slot");
    EngineHost &h = *host_;
    const SlotStatus st = h.h_status.ptr[s];  // filled by finished()
    const GraphImpl &g = *graphs_[sh.q.graph];
    if (sh.q.out) {
        const void *src = sh.q.kind == HYT_QUERY_SSSP ? static_cast<const void *>(h.ss[s].dist)
                                                      : static_cast<const void *>(h.pr[s].rank[st.iterations & 1]);
        if (g.inv.get()) {
            graph_emit(g, sh.q.out, src, stream_);  // back to the caller's ids
        } else {
            HYT_CUDA(cudaMemcpyAsync(sh.q.out, src, g.V * 4, cudaMemcpyDefault, stream_));
        }
    }
    if (res) {
        res->iterations = st.iterations;
        res->converged = st.converged;
        res->residual = st.residual;
        res->edges_processed = sh.q.kind == HYT_QUERY_SSSP ? st.edges : uint64_t(st.iterations) * g.E;
    }
    frontier_total += st.frontier;
    hub_need_ -= sh.hub;
    HYT_CUDA(cudaFreeAsync(sh.mem, stream_));
    in_use_ -= sh.bytes;
    --used_slots_;
    if (sh.running) --running_;
    sh = SlotHost{};
    h.slot[s] = Slot{kFree, 0, 0, 0};
    HYT_CUDA(cudaMemcpyAsync(h.d_slot.get() + s, &h.slot[s], sizeof(Slot), cudaMemcpyHostToDevice, stream_));
    while (hi_ > 0 && !slots_[hi_ - 1].used) --hi_;
    args_dirty_ = true;
}

void QueryEngine::reset() {
    cudaStreamSynchronize(stream_);
    (void)cudaGetLastError();
    EngineHost &h = *host_;
    for (uint32_t i = 0; i < cap_; ++i) {
        SlotHost &sh = slots_[i];
        if (sh.mem) cudaFreeAsync(sh.mem, stream_);
        sh = SlotHost{};
        h.slot[i] = Slot{kFree, 0, 0, 0};
    }
    cudaMemcpyAsync(h.d_slot.get(), h.slot.data(), cap_ * sizeof(Slot), cudaMemcpyHostToDevice, stream_);
    cudaStreamSynchronize(stream_);
    in_use_ = 0;
    hi_ = used_slots_ = running_ = 0;
    hub_need_ = 0;
    frontier_total = 0;
    args_dirty_ = true;
}

}  // namespace hyt

// ----------------------------------------------------------------- C ABI --
using namespace hyt;

namespace {

hyt_batch *batch_impl(hyt_batch *b) {
    if (!b || !b->engine) fail(HYT_E_INVALID, "batch handle is NULL");
    return b;
}

struct BatchTotals {
    uint32_t supersteps = 0, waves = 0, graph_launches = 0;
    uint64_t edges = 0, bytes = 0, peak_state = 0, kernels = 0;
};

// Admits queries in order while the state budget allows, runs each wave to
// completion, retires it; results[i] belongs to queries[i].
BatchTotals run_batch(hyt_batch *b, const hyt_query *q, uint32_t n, hyt_query_result *results, uint32_t flags) {
    QueryEngine &e = *b->engine;
    for (uint32_t i = 0; i < n; ++i) e.validate(q[i]);
    e.set_tuning(b->tuning);
    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH);
    BatchTotals t;
    const uint64_t l0 = e.launches();
    std::vector<hyt_query_result> local(n);
    uint32_t next = 0;
    while (next < n) {
        uint32_t admitted = 0;
        while (next < n) {
            if (e.admit(q[next], next) < 0) break;
            ++next;
            ++admitted;
        }
        if (admitted == 0) fail(HYT_E_OOM, "a query's state does not fit the batch state budget");
        t.peak_state = std::max(t.peak_state, e.bytes_in_use());
        t.supersteps += e.run_to_completion(use_graph);
        if (use_graph) ++t.graph_launches;
        for (const auto &f : e.finished()) e.retire(f.first, &local[f.second]);
        if (e.slots_in_use()) fail(HYT_E_INTERNAL, "batch ended with queries still running");
        ++t.waves;
    }
    HYT_CUDA(cudaStreamSynchronize(e.stream()));
    for (uint32_t i = 0; i < n; ++i) {
        const GraphImpl &g = *b->graphs[q[i].graph];
        t.edges += local[i].edges_processed;
        t.bytes += q[i].kind == HYT_QUERY_SSSP ? 12ull * local[i].edges_processed
                                               : uint64_t(local[i].iterations) * (8ull * g.E + 20ull * g.V);
        if (results) results[i] = local[i];
    }
    t.bytes += 16ull * e.frontier_total;
    e.frontier_total = 0;
    t.kernels = e.launches() - l0;
    return t;
}

}  // namespace

extern "C" {

int hyt_batch_create(hyt_graph *const *graphs, uint32_t num_graphs, const hyt_batch_options *options,
                     hyt_batch **out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        *out = nullptr;
        if (!graphs || num_graphs == 0) fail(HYT_E_INVALID, "a batch needs at least one graph");
        hyt_batch_options o = options_or_default(options);
        o.device = resolve_device(o.device);
        auto b = std::make_unique<hyt_batch>();
        b->device = o.device;
        for (uint32_t i = 0; i < num_graphs; ++i) {
            if (!graphs[i]) fail(HYT_E_INVALID, "graph handle is NULL");
            if (graphs[i]->impl.device != o.device) fail(HYT_E_INVALID, "every graph must live on the batch's device");
            b->graphs.push_back(&graphs[i]->impl);
            graph_vertex_map(graphs[i]->impl);  // queries map their sources on the host
        }
        HYT_CUDA(cudaSetDevice(o.device));
        HYT_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->tuning.delta_mult = o.tuning.delta_mult;
        if (o.tuning.hub_degree) b->tuning.hub_degree = o.tuning.hub_degree;
        b->tuning.ctas_per_sm = o.tuning.ctas_per_sm;
        b->flags = o.flags;
        try {
            b->engine = new QueryEngine(o.device, b->stream,
                                        o.state_budget_bytes ? o.state_budget_bytes : (uint64_t(16) << 30));
        } catch (...) {
            cudaStreamDestroy(b->stream);
            throw;
        }
        b->engine->set_graphs(b->graphs);
        *out = b.release();
    });
}

int hyt_batch_destroy(hyt_batch *b) {
    return guarded([&] {
        if (!b) return;
        cudaSetDevice(b->device);
        delete b->engine;
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
    });
}

int hyt_batch_set_tuning(hyt_batch *b, const hyt_batch_tuning *t) {
    return guarded([&] {
        batch_impl(b);
        if (!t) fail(HYT_E_INVALID, "tuning is NULL");
        b->tuning.delta_mult = t->delta_mult;
        b->tuning.hub_degree = t->hub_degree ? t->hub_degree : 64;
        b->tuning.ctas_per_sm = t->ctas_per_sm;
    });
}

int hyt_batch_run(hyt_batch *b, const hyt_query *queries, uint32_t num_queries, hyt_query_result *results,
                  hyt_batch_stats *stats) {
    return guarded([&] {
        batch_impl(b);
        if (!queries && num_queries) fail(HYT_E_INVALID, "queries is NULL");
        HYT_CUDA(cudaSetDevice(b->device));
        EventTimer total;
        total.start(b->stream);
        BatchTotals t;
        try {
            t = run_batch(b, queries, num_queries, results, b->flags);
        } catch (...) {
            b->engine->reset();
            throw;
        }
        total.stop(b->stream);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->device_ms = total.ms();
            stats->supersteps = t.supersteps;
            stats->waves = t.waves;
            stats->graph_launches = t.graph_launches;
            stats->kernel_launches = static_cast<uint32_t>(t.kernels);
            stats->edges_processed = t.edges;
            stats->algorithmic_bytes = t.bytes;
            stats->state_bytes = t.peak_state;
        }
    });
}

// Coordinate descent over the tuning knobs on an evenly spaced sample of
// the queries (at most 128, outputs dropped): bucket width first, then the
// hub threshold, then the persistent grid; each candidate is timed twice
// and scored by its faster run.  The choice is cached for the process per
// size class of the sample -- device, log2 of its mean graph edges and of
// its mean graph vertices, and its SSSP share in quarters -- so a later
// batch of the same class reuses it without timing anything.
namespace {
struct TuneClass {
    int device;
    int log_edges, log_vertices, sssp_quarters;
    bool operator<(const TuneClass &o) const {
        return std::tie(device, log_edges, log_vertices, sssp_quarters) <
               std::tie(o.device, o.log_edges, o.log_vertices, o.sssp_quarters);
    }
};
std::mutex g_tune_mu;
std::map<TuneClass, BatchTuning> g_tune_cache;

TuneClass tune_class(const hyt_batch *b, const std::vector<hyt_query> &sample) {
    double e = 0.0, v = 0.0;
    uint32_t sssp = 0;
    for (const hyt_query &q : sample) {
        const GraphImpl &g = *b->graphs[q.graph];
        e += static_cast<double>(g.E);
        v += static_cast<double>(g.V);
        sssp += q.kind == HYT_QUERY_SSSP ? 1u : 0u;
    }
    const double n = static_cast<double>(sample.size());
    return TuneClass{b->device, static_cast<int>(std::lround(std::log2(std::max(e / n, 1.0)))),
                     static_cast<int>(std::lround(std::log2(std::max(v / n, 1.0)))),
                     static_cast<int>(std::lround(4.0 * sssp / n))};
}
}  // namespace

int hyt_batch_autotune(hyt_batch *b, const hyt_query *queries, uint32_t num_queries, hyt_batch_tuning *chosen) {
    return guarded([&] {
        batch_impl(b);
        if (!queries || num_queries == 0) fail(HYT_E_INVALID, "autotune needs queries");
        HYT_CUDA(cudaSetDevice(b->device));
        const uint32_t m = std::min<uint32_t>(num_queries, 128);
        std::vector<hyt_query> sample(m);
        for (uint32_t i = 0; i < m; ++i) {
            sample[i] = queries[uint64_t(i) * num_queries / m];
            sample[i].out = nullptr;
        }
        for (const hyt_query &q : sample) b->engine->validate(q);
        auto report = [&](const BatchTuning &t) {
            if (chosen) {
                chosen->delta_mult = t.delta_mult;
                chosen->hub_degree = t.hub_degree;
                chosen->ctas_per_sm = t.ctas_per_sm;
            }
        };
        const TuneClass cls = tune_class(b, sample);
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            const auto it = g_tune_cache.find(cls);
            if (it != g_tune_cache.end()) {
                b->tuning = it->second;
                report(it->second);
                return;
            }
        }
        auto time_it = [&](const BatchTuning &t) {
            b->tuning = t;
            double best = 1e30;
            for (int rep = 0; rep < 2; ++rep) {
                EventTimer et;
                et.start(b->stream);
                try {
                    run_batch(b, sample.data(), m, nullptr, b->flags);
                } catch (...) {
                    b->engine->reset();
                    throw;
                }
                et.stop(b->stream);
                best = std::min(best, et.ms());
            }
            return best;
        };
        BatchTuning best = b->tuning;
        double best_ms = time_it(best);
        auto sweep = [&](auto set, std::initializer_list<uint32_t> values) {
            BatchTuning base = best;
            for (uint32_t v : values) {
                BatchTuning t = base;
                set(t, v);
                const double ms = time_it(t);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
        };
        sweep([](BatchTuning &t, uint32_t v) { t.delta_mult = v; }, {0u, 2u, 8u, 32u});
        sweep([](BatchTuning &t, uint32_t v) { t.hub_degree = v; }, {32u, 64u, 128u, 256u});
        sweep([](BatchTuning &t, uint32_t v) { t.ctas_per_sm = v; }, {0u, 1u, 2u});
        b->tuning = best;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[cls] = best;
        }
        report(best);
    });
}

}  // extern "C"
