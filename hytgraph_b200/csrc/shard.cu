// Vertex-range shards of a graph: one process per GPU, each computing one
// contiguous range of internal vertex ids, with the whole-graph per-vertex
// vectors exchanged by the caller's collective library between steps.
//
// Every process builds the same graph (same CSR, same flags), so all of
// them derive the same internal order, row tiles and shard bounds.
//
// PageRank (pull).  A shard is a run of whole row tiles, so its work list
// is a contiguous range of tile tasks plus the chunk tasks of the long rows
// that end those tiles.  A step runs the warp tasks of the single-GPU
// iteration (pagerank_core.cuh) over that range: it reads the whole-graph
// contribution vector and writes the rank and contribution of the range's
// rows.  Each row's sum has the association order of the single-GPU solve,
// so the ranks agree with hyt_pagerank except where the FP64 residual and
// dangling sums (atomics and the collective, in no fixed order) round
// differently in their last bits.
//
// SSSP (push shards).  Bellman-Ford rounds.  A round collects every owned
// vertex whose label dropped since it was last expanded (the shard's
// frontier) and counts its out-edges; the caller sums the count over the
// processes, so all shards take the same choice: a sparse frontier is
// pushed (its out-edges lower the labels of their heads in this process's
// copy of the whole label vector), a dense one (more than E / 4 out-edges,
// as hyt_sssp decides) makes every shard sweep its rows of the PULL bounds
// over the CSC instead.  The caller then min-reduces the label vector over
// all processes.  Labels are held as ordered keys (label XOR 0x80000000
// read as int32, so signed order is label order) because collective
// libraries reduce signed 32-bit integers.  The word after the labels is
// the idle flag: 1 when the shard's frontier was empty, so the same min
// reduction tells every process whether any shard still had work.  The
// fixed point is the unique shortest-path labelling, so the labels are
// bit-identical to hyt_sssp.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "graph.cuh"
#include "pagerank_core.cuh"
#include "scratch.cuh"
#include "solvers.cuh"
#include "sssp_core.cuh"

namespace hyt {

constexpr uint32_t kSegEdges = 256;           // out-edges per SSSP expansion segment
constexpr uint32_t kKeyBias = 0x80000000u;    // label -> ordered int32 key
constexpr int kExpandBatch = 4;               // 32-edge batches in flight per warp
constexpr uint32_t kShardPullDiv = 4;         // pull sweep when frontier out-edges > E / 4 (as hyt_sssp)

struct ShardImpl {
    GraphImpl *g = nullptr;
    uint32_t kind = 0, part = 0, parts = 0;
    uint32_t vb = 0, ve = 0;
    uint64_t edges = 0;  // in-edges (pull) or out-edges (push) of the range's rows
    // pull (and the pull sweeps of push shards): the range's PageRank tasks
    // and their long-row workspaces
    uint64_t chunk_begin = 0, chunk_end = 0, tile_begin = 0, tile_end = 0;
    GraphArray<float> partial;
    GraphArray<uint32_t> ticket;
    // push: label each owned vertex was last expanded with, expansion
    // segments, counters [0] expanded vertices of the round, [1] segments of
    // the round, [2] edges relaxed since init
    GraphArray<uint32_t> prev;
    GraphArray<uint4> segs;
    GraphArray<unsigned long long> ctr;
    uint32_t inf = HYT_DIST_INF_U32;
    // push: pull sweeps (rounds with a dense frontier) over this shard's
    // PageRank task range of the PULL bounds (fields above)
    bool pull_ok = false;
    uint64_t pull_edges = 0;
};

namespace {

using namespace prc;

// ---------------------------------------------------------------- PageRank

struct ShardTasks {
    uint64_t chunk_begin, chunk_end, tile_begin, tile_end;
    double dangling;  // whole-graph dangling mass of the iterate read
    double *sums;     // [0] += L1 change, [1] += dangling mass of the new iterate (range rows)
};

__global__ void __launch_bounds__(kPRThreads, 1) shard_pr_step_kernel(PRArgs a, PRBuffers b, ShardTasks t) {
    extern __shared__ __align__(16) float s_dyn[];
    __shared__ double s_red[32];

    const PRState ps = make_state(a, t.dangling);
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t n_chunks = t.chunk_end - t.chunk_begin;
    const uint64_t total = n_chunks + (t.tile_end - t.tile_begin);
    double res = 0.0, dang = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *s_hot = s_dyn;
    for (uint32_t i = threadIdx.x; i < a.num_hot; i += kPRThreads) s_hot[i] = b.ccur[a.hot_vertex[i]];
    __syncthreads();
    float *sv = s_dyn + a.num_hot + warp * (2 * a.tile_cost + 8);
    const uint64_t nwarps = uint64_t(gridDim.x) * (kPRThreads / 32);
    for (uint64_t task = uint64_t(blockIdx.x) * (kPRThreads / 32) + warp; task < total; task += nwarps) {
        if (task < n_chunks) {
            chunk_task<true>(a, ps, b, a.in_src, s_hot, t.chunk_begin + task, pol, lane, res, dang);
        } else {
            tile_task<true>(a, ps, b, a.in_src, s_hot, sv, t.tile_begin + (task - n_chunks), pol, lane, res, dang);
        }
    }
    const double bres = dev::block_sum(res, s_red);
    __syncthreads();
    const double bdang = dev::block_sum(dang, s_red);
    if (threadIdx.x == 0) {
        if (bres != 0.0) atomicAdd(t.sums, bres);
        if (bdang != 0.0) atomicAdd(t.sums + 1, bdang);
    }
}

// Initial iterate of every vertex (x_0 = 1/n, or the source indicator);
// sums[1] += dangling mass of the range's rows.
__global__ void shard_pr_init_kernel(const uint32_t *out_deg, uint32_t V, uint32_t vb, uint32_t ve,
                                     uint32_t personalized, uint32_t source, float *rank0, float *contrib0,
                                     double *sums) {
    __shared__ double s_red[32];
    const float uniform = __fdiv_rn(1.0f, static_cast<float>(V));
    double dang = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const float r0 = personalized ? (v == source ? 1.0f : 0.0f) : uniform;
        rank0[v] = r0;
        const uint32_t od = out_deg[v];
        contrib0[v] = od ? __fdiv_rn(r0, static_cast<float>(od)) : 0.0f;
        if (od == 0 && v >= vb && v < ve) dang += static_cast<double>(r0);
    }
    const double b = dev::block_sum(dang, s_red);
    if (threadIdx.x == 0 && b != 0.0) atomicAdd(sums + 1, b);
}

int shard_pr_grid() {
    static int grid = 0;
    if (grid == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaFuncSetAttribute(shard_pr_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shard_pr_step_kernel, kPRThreads,
                                                               kPRSmemMax));
        grid = sm_count() * std::max(per_sm, 1);
    }
    return grid;
}

// -------------------------------------------------------------------- SSSP

struct SSShard {
    const uint64_t *row_off;
    const uint32_t *cols;
    const uint32_t *weights;
    int32_t *keys;       // [V + 1]: ordered label keys + the idle flag
    uint32_t *prev;      // [ve - vb]
    uint4 *segs;         // (vertex, label, first edge, end edge)
    unsigned long long *ctr;
    const unsigned long long *frontier;  // out-edges of every shard's frontier this round
    uint64_t num_edges;
    uint32_t vb, ve, V;
    uint32_t pull_div;   // > 0: a round whose frontier has more than E / pull_div out-edges is a pull sweep
    uint32_t inf;
};

// The shard's pull sweep: its PageRank row tiles and long-row chunks over
// the CSC (in-sources tagged like PageRank's, weights in CSC order).
struct SSPull {
    const uint64_t *in_off;
    const uint32_t *in_src;
    const uint32_t *in_w;
    const uint32_t *tile_start;
    const LongRow *long_rows;
    const uint2 *chunk_tasks;
    const uint32_t *hot_vertex;
    uint64_t chunk_begin, chunk_end, tile_begin, tile_end;
    uint64_t edges;  // in-edges of the sweep's rows
    uint32_t num_hot, tile_cost;
};

// Same answer in every kernel of a round and on every shard (the count is
// the caller's sum over shards).
__device__ __forceinline__ bool shard_pull_round(const SSShard &a) {
    if (!a.pull_div) return false;
    const unsigned long long fe = *(volatile const unsigned long long *)a.frontier;
    return fe * a.pull_div > a.num_edges;
}

__global__ void shard_sssp_init_kernel(int32_t *keys, uint32_t V, uint32_t source, uint32_t inf, uint32_t *prev,
                                       uint32_t n_owned) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += stride)
        keys[v] = static_cast<int32_t>((v == source ? 0u : inf) ^ kKeyBias);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += stride) prev[i] = inf;
    if (blockIdx.x == 0 && threadIdx.x == 0) keys[V] = 0;
}

// Owned vertices whose label dropped since their last expansion: record the
// label and append the row as kSegEdges-edge segments (one warp-aggregated
// atomic per warp); ctr[3] += their out-edges.
__global__ void __launch_bounds__(256) shard_sssp_collect_kernel(SSShard a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t n = a.ve - a.vb;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i - lane < n; i += stride) {
        uint32_t v = 0, d = 0, nseg = 0;
        uint64_t lo = 0, hi = 0;
        bool act = false;
        if (i < n) {
            v = a.vb + static_cast<uint32_t>(i);
            d = static_cast<uint32_t>(a.keys[v]) ^ kKeyBias;
            if (d < a.prev[i]) {
                act = true;
                a.prev[i] = d;
                lo = a.row_off[v];
                hi = a.row_off[v + 1];
                nseg = static_cast<uint32_t>((hi - lo + kSegEdges - 1) / kSegEdges);
            }
        }
        const uint32_t amask = __ballot_sync(0xffffffffu, act);
        unsigned long long fe = hi - lo;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) fe += __shfl_xor_sync(0xffffffffu, fe, o);
        if (lane == 0 && fe) atomicAdd(&a.ctr[3], fe);
        uint32_t incl = nseg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= static_cast<uint32_t>(o)) incl += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        unsigned long long base = 0;
        if (lane == 0 && amask) atomicAdd(&a.ctr[0], static_cast<unsigned long long>(__popc(amask)));
        if (lane == 31 && tot) base = atomicAdd(&a.ctr[1], static_cast<unsigned long long>(tot));
        base = __shfl_sync(0xffffffffu, base, 31);
        const unsigned long long first = base + (incl - nseg);
        for (uint32_t k = 0; k < nseg; ++k) {
            const uint64_t e0 = lo + uint64_t(k) * kSegEdges;
            const uint64_t e1 = (e0 + kSegEdges < hi) ? e0 + kSegEdges : hi;
            a.segs[first + k] = make_uint4(v, d, static_cast<uint32_t>(e0), static_cast<uint32_t>(e1));
        }
    }
}

// A warp takes 32 segments, prefix-sums their lengths and walks the combined
// edge list 32 edges at a time (kExpandBatch batches in flight), finding
// each edge's segment with a 5-step shuffle search.  Thread 0 of block 0
// writes the idle flag from the round's expanded-vertex count; a pull round
// does nothing else here.
template <int WK>
__global__ void __launch_bounds__(256) shard_sssp_expand_kernel(SSShard a) {
    const uint64_t nseg = a.ctr[1];
    if (blockIdx.x == 0 && threadIdx.x == 0) a.keys[a.V] = a.ctr[0] ? 0 : 1;
    if (shard_pull_round(a)) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    unsigned long long relaxed = 0;
    for (uint64_t g0 = gw * 32; g0 < nseg; g0 += nw * 32) {
        const uint64_t i = g0 + lane;
        uint4 sg = make_uint4(0, 0, 0, 0);
        if (i < nseg) sg = a.segs[i];
        const uint32_t len = sg.w - sg.z;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= static_cast<uint32_t>(o)) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t excl = incl - len;
        relaxed += total;
        for (uint32_t base = 0; base < total; base += 32 * kExpandBatch) {
            uint32_t u[kExpandBatch], nd[kExpandBatch];
#pragma unroll
            for (int k = 0; k < kExpandBatch; ++k) {
                const uint32_t j = base + 32 * k + lane;
                uint32_t o = 0;  // last segment whose first combined index is <= j
#pragma unroll
                for (uint32_t step = 16; step; step >>= 1) {
                    const uint32_t ex = __shfl_sync(0xffffffffu, excl, o + step);
                    if (ex <= j) o += step;
                }
                const uint32_t lo = __shfl_sync(0xffffffffu, sg.z, o);
                const uint32_t d = __shfl_sync(0xffffffffu, sg.y, o);
                const uint32_t exo = __shfl_sync(0xffffffffu, excl, o);
                u[k] = 0;
                nd[k] = 0xFFFFFFFFu;  // above every label: no update
                if (j < total) {
                    const uint64_t e = uint64_t(lo) + (j - exo);
                    u[k] = dev::ld_stream(a.cols + e);
                    nd[k] = ssc::extend<WK>(d, ssc::edge_weight<WK>(a.weights, e));
                }
            }
            uint32_t cur[kExpandBatch];
#pragma unroll
            for (int k = 0; k < kExpandBatch; ++k)
                cur[k] = (nd[k] != 0xFFFFFFFFu) ? (static_cast<uint32_t>(__ldcg(a.keys + u[k])) ^ kKeyBias) : 0u;
#pragma unroll
            for (int k = 0; k < kExpandBatch; ++k)
                if (nd[k] < cur[k]) atomicMin(a.keys + u[k], static_cast<int32_t>(nd[k] ^ kKeyBias));
        }
    }
    if (lane == 0 && relaxed) atomicAdd(&a.ctr[2], relaxed);
}

// Candidate labels d[u] + w of in-edges [lo, hi) (infinity from unreached
// sources), 16 per lane in flight: ids and weights streamed, hot slots
// mapped to vertex ids through the CTA's table, labels gathered from L2.
constexpr int kShardPullBatch = 16;

template <int WK, class Sink>
__device__ __forceinline__ void shard_pull_span(const SSShard &a, const SSPull &p, const uint32_t *s_hot,
                                                uint64_t lo, uint64_t hi, uint64_t pol, int lane, Sink &&sink) {
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    for (uint32_t base = 0; base < n; base += 32 * kShardPullBatch) {
        uint32_t id[kShardPullBatch], w[kShardPullBatch], du[kShardPullBatch];
#pragma unroll
        for (int k = 0; k < kShardPullBatch; ++k) {
            const uint32_t i = base + 32 * k + lane;
            id[k] = (i < n) ? dev::ld_stream(p.in_src + lo + i) : 0u;
            w[k] = (i < n) ? ssc::edge_weight<WK>(p.in_w, lo + i) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kShardPullBatch; ++k)
            if (id[k] & kHotTag) id[k] = s_hot[id[k] & ~kHotTag];
#pragma unroll
        for (int k = 0; k < kShardPullBatch; ++k)
            du[k] = static_cast<uint32_t>(dev::ld_keep_u32(reinterpret_cast<const uint32_t *>(a.keys) + id[k], pol)) ^
                    kKeyBias;
#pragma unroll
        for (int k = 0; k < kShardPullBatch; ++k) {
            const uint32_t i = base + 32 * k + lane;
            if (i < n) sink(i, du[k] == a.inf ? a.inf : ssc::extend<WK>(du[k], w[k]));
        }
    }
}

__device__ __forceinline__ void shard_pull_relax(const SSShard &a, uint32_t r, uint32_t c) {
    if (c < (static_cast<uint32_t>(__ldcg(a.keys + r)) ^ kKeyBias))
        atomicMin(a.keys + r, static_cast<int32_t>(c ^ kKeyBias));
}

// Pull round: every row of the shard's sweep range takes the minimum over
// its in-edges of d[u] + w (the single-GPU sweep's task decomposition:
// merge-path tiles of short rows staged per warp, long rows in chunks whose
// minima meet in an atomic min).  Nothing in a push round.
template <int WK>
__global__ void __launch_bounds__(kPRThreads, 1) shard_sssp_pull_kernel(SSShard a, SSPull p) {
    extern __shared__ __align__(16) uint32_t s_pull[];
    if (!shard_pull_round(a)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *s_hot = s_pull;
    for (uint32_t i = threadIdx.x; i < p.num_hot; i += blockDim.x) s_hot[i] = p.hot_vertex[i];
    __syncthreads();
    uint32_t *sv = s_pull + p.num_hot + warp * (2 * p.tile_cost + 8);
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t n_chunks = p.chunk_end - p.chunk_begin;
    const uint64_t total = n_chunks + (p.tile_end - p.tile_begin);
    const uint64_t nwarps = uint64_t(gridDim.x) * (kPRThreads / 32);
    for (uint64_t task = uint64_t(blockIdx.x) * (kPRThreads / 32) + warp; task < total; task += nwarps) {
        if (task < n_chunks) {
            const uint2 t = p.chunk_tasks[p.chunk_begin + task];
            const LongRow L = p.long_rows[t.x];
            const uint64_t rb = p.in_off[L.row], re = p.in_off[L.row + 1];
            const uint64_t lo = rb + uint64_t(t.y) * kLongChunk;
            const uint64_t hi = (lo + kLongChunk < re) ? lo + kLongChunk : re;
            uint32_t best = a.inf;
            shard_pull_span<WK>(a, p, s_hot, lo, hi, pol, lane, [&](uint32_t, uint32_t c) { best = min(best, c); });
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (lane == 0) shard_pull_relax(a, L.row, best);
        } else {
            const uint64_t k = p.tile_begin + (task - n_chunks);
            const uint32_t r0 = p.tile_start[k], r1 = p.tile_start[k + 1];
            if (r0 == r1) continue;
            const uint64_t last_b = p.in_off[r1 - 1], last_e = p.in_off[r1];
            const uint32_t rl = (last_e - last_b >= p.tile_cost) ? r1 - 1 : r1;  // long last row is chunked
            const uint64_t e0 = p.in_off[r0];
            const uint64_t e1 = (rl == r1) ? last_e : last_b;
            shard_pull_span<WK>(a, p, s_hot, e0, e1, pol, lane, [&](uint32_t i, uint32_t c) { sv[i] = c; });
            __syncwarp();
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t r = rb + lane;
                const bool active = r < rl;
                const uint64_t lo = active ? p.in_off[r] : 0;
                const uint64_t hi = active ? p.in_off[r + 1] : 0;
                if (active && hi - lo < 64) {
                    uint32_t best = a.inf;
                    for (uint64_t x = lo; x < hi; ++x) best = min(best, sv[x - e0]);
                    shard_pull_relax(a, r, best);
                }
                uint32_t big = __ballot_sync(0xffffffffu, active && (hi - lo >= 64));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, hi, src);
                    uint32_t best = a.inf;
                    for (uint64_t x = bb + lane; x < ee; x += 32) best = min(best, sv[x - e0]);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
                    if (lane == 0) shard_pull_relax(a, rb + src, best);
                }
            }
            __syncwarp();
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.edges) atomicAdd(&a.ctr[2], static_cast<unsigned long long>(p.edges));
}

__global__ void shard_keys_to_labels_kernel(const int32_t *keys, uint64_t V, uint32_t *labels) {
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x)
        labels[v] = static_cast<uint32_t>(keys[v]) ^ kKeyBias;
}

SSShard sssp_view(ShardImpl &sh, int32_t *keys) {
    GraphImpl &g = *sh.g;
    SSShard a{};
    a.row_off = g.row_offsets.get();
    a.cols = g.cols.get();
    a.weights = g.weights.get();
    a.keys = keys;
    a.prev = sh.prev.get();
    a.segs = sh.segs.get();
    a.ctr = sh.ctr.get();
    a.frontier = sh.ctr.get() + 3;
    a.num_edges = g.E;
    a.vb = sh.vb;
    a.ve = sh.ve;
    a.V = static_cast<uint32_t>(g.V);
    a.pull_div = 0;
    a.inf = sh.inf;
    return a;
}

SSPull pull_view(const ShardImpl &sh) {
    const GraphImpl &g = *sh.g;
    SSPull p{};
    p.in_off = g.in_offsets.get();
    p.in_src = g.in_sources.get();
    p.in_w = g.in_weights.get();
    p.tile_start = g.tile_start.get();
    p.long_rows = g.long_rows.get();
    p.chunk_tasks = g.chunk_tasks.get();
    p.hot_vertex = g.hot_vertex.get();
    p.chunk_begin = sh.chunk_begin;
    p.chunk_end = sh.chunk_end;
    p.tile_begin = sh.tile_begin;
    p.tile_end = sh.tile_end;
    p.edges = sh.pull_edges;
    p.num_hot = g.num_hot;
    p.tile_cost = g.tile_cost;
    return p;
}

cudaStream_t stream_of(const ShardImpl &sh, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : sh.g->stream;
}

// Host copy of a device array.
template <class T>
std::vector<T> download(const T *p, size_t n, cudaStream_t s) {
    std::vector<T> h(n);
    if (n) {
        HYT_CUDA(cudaMemcpyAsync(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
    }
    return h;
}

// Smallest index i in [0, n] with cost(i) >= target (cost non-decreasing).
template <class F>
uint64_t lower_index(uint64_t n, uint64_t target, F &&cost) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (cost(mid) >= target) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    return lo;
}

}  // namespace

// Work = rows + edges; cut p is the first admissible vertex at which the
// prefix work reaches p/parts of the total.  Pull cuts fall on row tiles.
void shard_bounds(GraphImpl &g, uint32_t kind, uint32_t parts, uint32_t *bounds) {
    if (parts == 0) fail(HYT_E_INVALID, "shard bounds need at least one part");
    const cudaStream_t s = g.stream;
    const uint64_t V = g.V;
    const uint64_t total = V + g.E;
    bounds[0] = 0;
    bounds[parts] = static_cast<uint32_t>(V);
    if (kind == HYT_SHARD_PULL) {
        if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "pull shards need a graph created with HYT_GRAPH_PULL");
        const std::vector<uint32_t> ts = download(g.tile_start.get(), g.num_tiles + 1, s);
        const std::vector<uint64_t> off = download(g.in_offsets.get(), V + 1, s);
        for (uint32_t p = 1; p < parts; ++p) {
            const uint64_t target = (total * p + parts - 1) / parts;
            const uint64_t k = lower_index(g.num_tiles, target, [&](uint64_t t) { return off[ts[t]] + ts[t]; });
            bounds[p] = std::max(ts[k], bounds[p - 1]);
        }
    } else if (kind == HYT_SHARD_PUSH) {
        if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "push shards need a graph created with HYT_GRAPH_PUSH");
        const std::vector<uint64_t> off = download(g.row_offsets.get(), V + 1, s);
        for (uint32_t p = 1; p < parts; ++p) {
            const uint64_t target = (total * p + parts - 1) / parts;
            const uint64_t v = lower_index(V, target, [&](uint64_t x) { return off[x] + x; });
            bounds[p] = std::max(static_cast<uint32_t>(v), bounds[p - 1]);
        }
    } else {
        fail(HYT_E_INVALID, "shard kind must be HYT_SHARD_PULL or HYT_SHARD_PUSH");
    }
}

namespace {

// PageRank task range of the rows [vb, ve) (bounds on row tiles) into sh's
// tile / chunk fields; returns the rows' in-edges.
uint64_t pull_tasks(GraphImpl &g, uint32_t vb, uint32_t ve, ShardImpl &sh) {
    const cudaStream_t s = g.stream;
    const std::vector<uint32_t> ts = download(g.tile_start.get(), g.num_tiles + 1, s);
    auto tile_of = [&](uint32_t v) -> uint64_t {
        const auto it = std::lower_bound(ts.begin(), ts.end(), v);
        if (it == ts.end() || *it != v) fail(HYT_E_INVALID, "pull shard bounds must fall on row tiles (hyt_shard_bounds)");
        return static_cast<uint64_t>(it - ts.begin());
    };
    // the first tile starting at each bound: neighbouring shards split the
    // tile list without overlap even where empty tiles repeat a start
    sh.tile_begin = tile_of(vb);
    sh.tile_end = tile_of(ve);
    // long rows end tiles, so the range's long rows are those with a row in
    // [vb, ve); their chunk tasks are one contiguous run
    const std::vector<LongRow> lr = download(g.long_rows.get(), g.num_long, s);
    const std::vector<uint2> ct = download(g.chunk_tasks.get(), g.num_chunks, s);
    uint64_t li = 0;
    while (li < lr.size() && lr[li].row < vb) ++li;
    uint64_t lj = li;
    while (lj < lr.size() && lr[lj].row < ve) ++lj;
    for (uint64_t k = li; k < lj; ++k) {
        if (k + 1 < lj && lr[k + 1].first_chunk != lr[k].first_chunk + lr[k].num_chunks)
            fail(HYT_E_INTERNAL, "long-row chunk tasks are not contiguous");
        for (uint32_t j = 0; j < lr[k].num_chunks; ++j) {
            const uint64_t c = uint64_t(lr[k].first_chunk) + j;
            if (c >= ct.size() || ct[c].x != k || ct[c].y != j)
                fail(HYT_E_INTERNAL, "long-row chunk tasks are not in long-row order");
        }
    }
    sh.chunk_begin = (li < lj) ? lr[li].first_chunk : 0;
    sh.chunk_end = (li < lj) ? uint64_t(lr[lj - 1].first_chunk) + lr[lj - 1].num_chunks : 0;
    uint64_t e[2] = {0, 0};
    HYT_CUDA(cudaMemcpyAsync(&e[0], g.in_offsets.get() + vb, 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaMemcpyAsync(&e[1], g.in_offsets.get() + ve, 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    return e[1] - e[0];
}

}  // namespace

void shard_create(GraphImpl &g, uint32_t kind, const uint32_t *bounds, uint32_t parts, uint32_t part,
                  ShardImpl &sh) {
    if (!bounds) fail(HYT_E_INVALID, "bounds is NULL");
    if (parts == 0 || part >= parts) fail(HYT_E_INVALID, "shard part must be < parts");
    if (bounds[0] != 0 || bounds[parts] != g.V) fail(HYT_E_INVALID, "shard bounds must run from 0 to num_vertices");
    for (uint32_t p = 0; p < parts; ++p)
        if (bounds[p] > bounds[p + 1]) fail(HYT_E_INVALID, "shard bounds must be non-decreasing");
    const cudaStream_t s = g.stream;
    sh.g = &g;
    sh.kind = kind;
    sh.part = part;
    sh.parts = parts;
    sh.vb = bounds[part];
    sh.ve = bounds[part + 1];
    if (kind == HYT_SHARD_PULL) {
        if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "pull shards need a graph created with HYT_GRAPH_PULL");
        sh.edges = pull_tasks(g, sh.vb, sh.ve, sh);
        sh.partial.allocate(2 * std::max<uint64_t>(g.num_chunks, 1));
        sh.ticket.allocate(std::max<uint64_t>(g.num_long, 1));
        HYT_CUDA(cudaMemsetAsync(sh.ticket.get(), 0, sh.ticket.count * sizeof(uint32_t), s));
        HYT_CUDA(cudaStreamSynchronize(s));
    } else if (kind == HYT_SHARD_PUSH) {
        if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "push shards need a graph created with HYT_GRAPH_PUSH");
        if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
        uint64_t e[2] = {0, 0};
        HYT_CUDA(cudaMemcpyAsync(&e[0], g.row_offsets.get() + sh.vb, 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(&e[1], g.row_offsets.get() + sh.ve, 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        sh.edges = e[1] - e[0];
        const uint64_t n = sh.ve - sh.vb;
        // every expanded vertex yields ceil(deg / kSegEdges) <= deg / kSegEdges + 1 segments
        const uint64_t cap = n + sh.edges / kSegEdges + 1;
        sh.prev.allocate(std::max<uint64_t>(n, 1));
        sh.segs.allocate(cap);
        sh.ctr.allocate(4);
        HYT_CUDA(cudaMemsetAsync(sh.ctr.get(), 0, 4 * sizeof(unsigned long long), s));
        HYT_CUDA(cudaStreamSynchronize(s));
        sh.inf = (g.weight_kind == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
        // Pull sweeps cover the rows of this shard's part of the PULL bounds
        // (a second partition of the same vertices, derived identically by
        // every process); they need the CSC and its weights.
        if ((g.flags & HYT_GRAPH_PULL) && (g.weight_kind == HYT_WEIGHTS_NONE || g.in_weights.get()) && g.E > 0) {
            std::vector<uint32_t> pb(parts + 1);
            shard_bounds(g, HYT_SHARD_PULL, parts, pb.data());
            sh.pull_edges = pull_tasks(g, pb[part], pb[part + 1], sh);
            sh.pull_ok = true;
        }
    } else {
        fail(HYT_E_INVALID, "shard kind must be HYT_SHARD_PULL or HYT_SHARD_PUSH");
    }
}

namespace {

void check_pr_args(const ShardImpl &sh, const hyt_shard_pagerank &p) {
    if (sh.kind != HYT_SHARD_PULL) fail(HYT_E_INVALID, "PageRank runs on pull shards");
    if (!p.rank[0] || !p.rank[1] || !p.contrib[0] || !p.contrib[1] || !p.sums)
        fail(HYT_E_INVALID, "shard PageRank vectors must be non-NULL device pointers");
    if (!(p.damping >= 0.0f && p.damping < 1.0f)) fail(HYT_E_INVALID, "PageRank damping_factor must be in [0, 1)");
    if (p.personalized && p.source >= sh.g->V) fail(HYT_E_INVALID, "personalized PageRank source vertex is out of range");
}

}  // namespace

void shard_pagerank_init(ShardImpl &sh, const hyt_shard_pagerank &p) {
    check_pr_args(sh, p);
    GraphImpl &g = *sh.g;
    const cudaStream_t s = stream_of(sh, p.stream);
    const uint32_t src = p.personalized ? graph_vertex(g, p.source, s) : 0u;
    HYT_CUDA(cudaMemsetAsync(p.sums, 0, 2 * sizeof(double), s));
    HYT_CUDA(cudaMemsetAsync(sh.ticket.get(), 0, sh.ticket.count * sizeof(uint32_t), s));
    shard_pr_init_kernel<<<grid_for(g.V, 256, 148 * 8), 256, 0, s>>>(
        g.out_degree.get(), static_cast<uint32_t>(g.V), sh.vb, sh.ve, p.personalized ? 1u : 0u, src, p.rank[0],
        p.contrib[0], p.sums);
    HYT_CUDA(cudaGetLastError());
}

void shard_pagerank_step(ShardImpl &sh, const hyt_shard_pagerank &p, uint32_t it, double dangling) {
    check_pr_args(sh, p);
    GraphImpl &g = *sh.g;
    const cudaStream_t s = stream_of(sh, p.stream);
    HYT_CUDA(cudaMemsetAsync(p.sums, 0, 2 * sizeof(double), s));
    const uint64_t tasks = (sh.chunk_end - sh.chunk_begin) + (sh.tile_end - sh.tile_begin);
    if (tasks == 0) return;
    PRArgs a{};
    a.in_off = g.in_offsets.get();
    a.in_src = g.in_sources.get();
    a.out_deg = g.out_degree.get();
    a.tile_start = g.tile_start.get();
    a.long_rows = g.long_rows.get();
    a.chunk_tasks = g.chunk_tasks.get();
    a.hot_vertex = g.hot_vertex.get();
    a.num_hot = g.num_hot;
    a.tile_cost = g.tile_cost;
    a.partial = reinterpret_cast<float2 *>(sh.partial.get());
    a.ticket = sh.ticket.get();
    a.num_tiles = g.num_tiles;
    a.num_chunks = static_cast<uint32_t>(g.num_chunks);
    a.V = static_cast<uint32_t>(g.V);
    a.damping = p.damping;
    a.base = p.personalized ? 0.0f : (1.0f - p.damping) / static_cast<float>(g.V);
    a.source = p.personalized ? graph_vertex(g, p.source, s) : 0u;
    a.personalized = p.personalized ? 1u : 0u;
    PRBuffers b;
    b.cur = p.rank[it & 1];
    b.nxt = p.rank[(it + 1) & 1];
    b.ccur = p.contrib[it & 1];
    b.cnxt = p.contrib[(it + 1) & 1];
    const ShardTasks t{sh.chunk_begin, sh.chunk_end, sh.tile_begin, sh.tile_end, dangling, p.sums};
    const uint64_t want = (tasks + kPRThreads / 32 - 1) / (kPRThreads / 32);
    const int grid = static_cast<int>(std::min<uint64_t>(shard_pr_grid(), want));
    shard_pr_step_kernel<<<grid, kPRThreads, pr_shared_bytes(g.num_hot, g.tile_cost), s>>>(a, b, t);
    HYT_CUDA(cudaGetLastError());
}

void shard_sssp_init(ShardImpl &sh, const hyt_shard_sssp &p) {
    if (sh.kind != HYT_SHARD_PUSH) fail(HYT_E_INVALID, "SSSP runs on push shards");
    if (!p.keys) fail(HYT_E_INVALID, "shard SSSP keys must be a non-NULL device pointer");
    GraphImpl &g = *sh.g;
    if (p.source >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    const cudaStream_t s = stream_of(sh, p.stream);
    const uint32_t src = graph_vertex(g, p.source, s);
    HYT_CUDA(cudaMemsetAsync(sh.ctr.get(), 0, 4 * sizeof(unsigned long long), s));
    shard_sssp_init_kernel<<<grid_for(g.V + 1, 256, 148 * 8), 256, 0, s>>>(
        p.keys, static_cast<uint32_t>(g.V), src, sh.inf, sh.prev.get(), sh.ve - sh.vb);
    HYT_CUDA(cudaGetLastError());
}

namespace {

void check_ss_args(const ShardImpl &sh, const hyt_shard_sssp &p) {
    if (sh.kind != HYT_SHARD_PUSH) fail(HYT_E_INVALID, "SSSP runs on push shards");
    if (!p.keys) fail(HYT_E_INVALID, "shard SSSP keys must be a non-NULL device pointer");
}

int pull_grid_for(const void *fn) {
    int per_sm = 0;
    HYT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kPRSmemMax)));
    HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPRThreads, kPRSmemMax));
    return sm_count() * std::max(per_sm, 1);
}

template <int WK>
void launch_relax(const ShardImpl &sh, const SSShard &a, cudaStream_t s) {
    shard_sssp_expand_kernel<WK><<<static_cast<unsigned>(sm_count()) * 8u, 256, 0, s>>>(a);
    HYT_CUDA(cudaGetLastError());
    if (!a.pull_div) return;
    const SSPull p = pull_view(sh);
    const uint64_t tasks = (p.chunk_end - p.chunk_begin) + (p.tile_end - p.tile_begin);
    if (tasks == 0) return;
    static const int full = pull_grid_for(reinterpret_cast<const void *>(shard_sssp_pull_kernel<WK>));
    const uint64_t want = (tasks + kPRThreads / 32 - 1) / (kPRThreads / 32);
    const int grid = static_cast<int>(std::min<uint64_t>(full, want));
    shard_sssp_pull_kernel<WK><<<grid, kPRThreads, pr_shared_bytes(p.num_hot, p.tile_cost), s>>>(a, p);
    HYT_CUDA(cudaGetLastError());
}

}  // namespace

void shard_sssp_collect(ShardImpl &sh, const hyt_shard_sssp &p) {
    check_ss_args(sh, p);
    const cudaStream_t s = stream_of(sh, p.stream);
    HYT_CUDA(cudaMemsetAsync(sh.ctr.get(), 0, 2 * sizeof(unsigned long long), s));
    HYT_CUDA(cudaMemsetAsync(sh.ctr.get() + 3, 0, sizeof(unsigned long long), s));
    const SSShard a = sssp_view(sh, p.keys);
    const uint64_t n = sh.ve - sh.vb;
    if (n) {
        shard_sssp_collect_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(a);
        HYT_CUDA(cudaGetLastError());
    }
    if (p.frontier_edges)
        HYT_CUDA(cudaMemcpyAsync(p.frontier_edges, sh.ctr.get() + 3, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
}

// Pull sweeps need one decision for all shards: the caller's summed
// frontier count, or a single shard deciding alone.
void shard_sssp_relax(ShardImpl &sh, const hyt_shard_sssp &p) {
    check_ss_args(sh, p);
    GraphImpl &g = *sh.g;
    const cudaStream_t s = stream_of(sh, p.stream);
    SSShard a = sssp_view(sh, p.keys);
    if (p.frontier_edges) a.frontier = reinterpret_cast<const unsigned long long *>(p.frontier_edges);
    const bool shared_decision = p.frontier_edges != nullptr || sh.parts == 1;
    a.pull_div = (sh.pull_ok && shared_decision) ? kShardPullDiv : 0u;
    switch (g.weight_kind) {
        case HYT_WEIGHTS_NONE: launch_relax<HYT_WEIGHTS_NONE>(sh, a, s); break;
        case HYT_WEIGHTS_U32: launch_relax<HYT_WEIGHTS_U32>(sh, a, s); break;
        case HYT_WEIGHTS_F32: launch_relax<HYT_WEIGHTS_F32>(sh, a, s); break;
        default: fail(HYT_E_INTERNAL, "unknown weight kind");
    }
}

void shard_sssp_round(ShardImpl &sh, const hyt_shard_sssp &p) {
    hyt_shard_sssp q = p;
    q.frontier_edges = nullptr;
    shard_sssp_collect(sh, q);
    shard_sssp_relax(sh, q);
}

void shard_sssp_labels(ShardImpl &sh, const int32_t *keys, uint32_t *out, void *stream) {
    if (sh.kind != HYT_SHARD_PUSH) fail(HYT_E_INVALID, "SSSP labels come from push shards");
    if (!keys || !out) fail(HYT_E_INVALID, "keys and out must be non-NULL");
    GraphImpl &g = *sh.g;
    const cudaStream_t s = stream_of(sh, stream);
    Scratch<uint32_t> lab(g.V, s);
    shard_keys_to_labels_kernel<<<grid_for(g.V, 256), 256, 0, s>>>(keys, g.V, lab.get());
    HYT_CUDA(cudaGetLastError());
    graph_emit(g, out, lab.get(), s);
    HYT_CUDA(cudaStreamSynchronize(s));
}

void shard_emit(ShardImpl &sh, const void *src, void *dst, void *stream) {
    if (!src || !dst) fail(HYT_E_INVALID, "src and dst must be non-NULL");
    const cudaStream_t s = stream_of(sh, stream);
    graph_emit(*sh.g, dst, src, s);
    HYT_CUDA(cudaStreamSynchronize(s));
}

void shard_info(const ShardImpl &sh, hyt_shard_info *out) {
    std::memset(out, 0, sizeof(*out));
    out->kind = sh.kind;
    out->part = sh.part;
    out->parts = sh.parts;
    out->vertex_begin = sh.vb;
    out->vertex_end = sh.ve;
    out->num_vertices = sh.g->V;
    out->edges = sh.edges;
    if (sh.kind == HYT_SHARD_PULL) {
        out->tasks = (sh.chunk_end - sh.chunk_begin) + (sh.tile_end - sh.tile_begin);
    } else {
        unsigned long long c[4] = {0, 0, 0, 0};
        HYT_CUDA(cudaMemcpyAsync(c, sh.ctr.get(), sizeof(c), cudaMemcpyDeviceToHost, sh.g->stream));
        HYT_CUDA(cudaStreamSynchronize(sh.g->stream));
        out->edges_relaxed = c[2];
    }
}

}  // namespace hyt

// extern "C" entry points of the shard API (declared in include/hyt/capi.h).
struct hyt_shard {
    hyt::ShardImpl impl;
};

using namespace hyt;

namespace {

ShardImpl &shard_impl(hyt_shard *s) {
    if (!s) fail(HYT_E_INVALID, "shard handle is NULL");
    HYT_CUDA(cudaSetDevice(s->impl.g->device));
    return s->impl;
}

GraphImpl &graph_impl(hyt_graph *g) {
    if (!g) fail(HYT_E_INVALID, "graph handle is NULL");
    HYT_CUDA(cudaSetDevice(g->impl.device));
    return g->impl;
}

}  // namespace

extern "C" {

int hyt_shard_bounds(hyt_graph *graph, uint32_t kind, uint32_t parts, uint32_t *bounds) {
    return guarded([&] {
        if (!bounds) fail(HYT_E_INVALID, "bounds is NULL");
        shard_bounds(graph_impl(graph), kind, parts, bounds);
    });
}

int hyt_shard_create(hyt_graph *graph, uint32_t kind, const uint32_t *bounds, uint32_t parts, uint32_t part,
                     hyt_shard **out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        *out = nullptr;
        GraphImpl &g = graph_impl(graph);
        std::unique_ptr<hyt_shard> s(new hyt_shard);
        shard_create(g, kind, bounds, parts, part, s->impl);
        *out = s.release();
    });
}

int hyt_shard_destroy(hyt_shard *shard) {
    // Touches only the shard's own arrays (each frees on the device it was
    // allocated on), so it is safe after the graph was destroyed.
    return guarded([&] { delete shard; });
}

int hyt_shard_get_info(hyt_shard *shard, hyt_shard_info *out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        shard_info(shard_impl(shard), out);
    });
}

int hyt_shard_pagerank_init(hyt_shard *shard, const hyt_shard_pagerank *args) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_pagerank_init(shard_impl(shard), *args);
    });
}

int hyt_shard_pagerank_step(hyt_shard *shard, const hyt_shard_pagerank *args, uint32_t iteration, double dangling) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_pagerank_step(shard_impl(shard), *args, iteration, dangling);
    });
}

int hyt_shard_sssp_init(hyt_shard *shard, const hyt_shard_sssp *args) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_sssp_init(shard_impl(shard), *args);
    });
}

int hyt_shard_sssp_collect(hyt_shard *shard, const hyt_shard_sssp *args) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_sssp_collect(shard_impl(shard), *args);
    });
}

int hyt_shard_sssp_relax(hyt_shard *shard, const hyt_shard_sssp *args) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_sssp_relax(shard_impl(shard), *args);
    });
}

int hyt_shard_sssp_round(hyt_shard *shard, const hyt_shard_sssp *args) {
    return guarded([&] {
        if (!args) fail(HYT_E_INVALID, "args is NULL");
        shard_sssp_round(shard_impl(shard), *args);
    });
}

int hyt_shard_sssp_labels(hyt_shard *shard, const int32_t *keys, uint32_t *out, void *stream) {
    return guarded([&] { shard_sssp_labels(shard_impl(shard), keys, out, stream); });
}

int hyt_shard_emit(hyt_shard *shard, const void *values, void *out, void *stream) {
    return guarded([&] { shard_emit(shard_impl(shard), values, out, stream); });
}

}  // extern "C"
