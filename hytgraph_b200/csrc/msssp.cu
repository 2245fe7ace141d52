// Multi-source SSSP: up to 8 sources on one graph in one solve
// (hyt_sssp_multi).
//
// Every source keeps the single-source definition (hyt_sssp; the
// reference's sssp_cpu fixed point, src/algorithms/sssp.cpp:109-234): the
// labels are the unique shortest-path distances, reached by any
// label-correcting schedule, so each lane is bit-identical to hyt_sssp from
// its source.
//
// The 8 labels of a vertex sit together in one 32-byte row (lanes beyond
// the query count stay at infinity), so work is shared across the sources:
//   push round -- the union frontier (vertices whose label dropped in any
//                 lane) is expanded once; per out-edge one id, one weight
//                 and one 32-byte label row of the head, then an atomicMin
//                 only for lanes that improve.  Rows of >= kHubDegree edges
//                 become 512-edge warp tasks of a second kernel.
//   pull sweep -- when the frontier's out-edges exceed E / 4, every row
//                 takes, per lane, the minimum of d[u] + w over its
//                 in-edges: one id and one 32-byte label row per in-edge
//                 for all lanes, 4 label rows in flight per thread; ids
//                 read in place on the default 512-unit tiles, or staged
//                 by bulk copies (stage.cuh) on 256-unit tiles
//                 (HYT_STAGED=1).  Tile rows are written with plain stores
//                 (one writer per row during a sweep).
// Per edge the memory traffic is about that of one single-source
// relaxation, whatever the number of lanes; the rounds are those of the
// deepest source.  Rounds run as a CUDA-graph conditional while-loop.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bulk.cuh"
#include "common.cuh"
#include "graph.cuh"
#include "scratch.cuh"
#include "solvers.cuh"
#include "sssp_core.cuh"
#include "stage.cuh"

namespace hyt {
namespace {

using ssc::extend;
using ssc::kHubChunk;
using ssc::kHubDegree;

constexpr int kML = 8;             // labels per vertex row (32 bytes)
constexpr int kMSThreads = 256;    // push kernels
constexpr int kMPThreads = stage::kStageThreads;   // pull sweep (one CTA per SM)

struct MSHeader {
    uint32_t round, done, converged, error;
    uint32_t qsize[2];
    uint32_t hub_count;
    uint32_t max_rounds;
    unsigned long long relaxations;     // push: frontier out-edges; pull: E per sweep
    unsigned long long frontier_total;  // frontier vertices expanded
    unsigned long long frontier_edges;  // out-edges of this round's frontier
    uint32_t pull_rounds, close_ticket;  // close_ticket: blocks of the round-close kernel finished
    unsigned long long frontier_edges_next;  // out-edges of the next frontier, summed at round close
};

struct MSArgs {
    const uint64_t *row_off;
    const uint32_t *cols;
    const uint32_t *weights;
    uint32_t *dist;  // [V][kML]
    uint32_t *stamp;
    uint32_t *queue[2];
    uint2 *hubs;
    MSHeader *hdr;
    uint32_t V, k, inf, use_cond;
    cudaGraphConditionalHandle cond;
    uint32_t pull_div;
    uint64_t num_edges;
    uint32_t sources[kML];
    // pull side (CSC, weights in CSC order, staged task list)
    const uint64_t *in_off;
    const uint32_t *in_src;
    const uint32_t *in_w;
    const uint32_t *hot_vertex;
    const LongRow *long_rows;
    const uint4 *tasks;
    uint64_t num_tasks;
    uint32_t num_hot;
};

struct Row8 {
    uint32_t d[kML];
};

__device__ __forceinline__ Row8 load_row(const uint32_t *dist, uint32_t v) {
    const uint4 *p = reinterpret_cast<const uint4 *>(dist + size_t(v) * kML);
    const uint4 a = __ldcg(p), b = __ldcg(p + 1);
    return Row8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}

// Label row read through L2 with an evict-last policy (pull gathers).
__device__ __forceinline__ Row8 load_row_keep(const uint32_t *dist, uint32_t v, uint64_t pol) {
    const uint32_t *p = dist + size_t(v) * kML;
    Row8 r;
    asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(r.d[0]), "=r"(r.d[1]), "=r"(r.d[2]), "=r"(r.d[3])
                 : "l"(p), "l"(pol));
    asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(r.d[4]), "=r"(r.d[5]), "=r"(r.d[6]), "=r"(r.d[7])
                 : "l"(p + 4), "l"(pol));
    return r;
}

__device__ __forceinline__ bool pull_round(const MSArgs &a) {
    if (!a.pull_div) return false;
    const unsigned long long fe = *(volatile const unsigned long long *)&a.hdr->frontier_edges;
    return fe * a.pull_div > a.num_edges;
}

struct View {
    uint32_t r, qn, next_stamp;
    const uint32_t *q;
    uint32_t *qnext, *qnext_size;
};

__device__ __forceinline__ View view(const MSArgs &a) {
    View w;
    w.r = *(volatile const uint32_t *)&a.hdr->round;
    const uint32_t odd = w.r & 1;
    w.qn = *(volatile const uint32_t *)(odd ? &a.hdr->qsize[1] : &a.hdr->qsize[0]);
    w.q = odd ? a.queue[1] : a.queue[0];
    w.qnext = odd ? a.queue[0] : a.queue[1];
    w.qnext_size = odd ? &a.hdr->qsize[0] : &a.hdr->qsize[1];
    w.next_stamp = w.r + 1;
    return w;
}

// Relaxes edge (u -> v, weight w) in every lane with u's labels du; true
// when some lane of v improved and v joins the next frontier now.
template <int WK>
__device__ __forceinline__ bool relax_row(const MSArgs &a, const View &w, const Row8 &du, uint32_t v, uint32_t wt) {
    const Row8 dv = load_row(a.dist, v);
    bool improved = false;
#pragma unroll
    for (int l = 0; l < kML; ++l) {
        if (l >= static_cast<int>(a.k) || du.d[l] == a.inf) continue;
        const uint32_t c = extend<WK>(du.d[l], wt);
        if (c < dv.d[l]) improved |= c < atomicMin(a.dist + size_t(v) * kML + l, c);
    }
    return improved && atomicExch(a.stamp + v, w.next_stamp) != w.next_stamp;
}

__global__ void ms_init_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    const uint64_t n = uint64_t(a.V) * kML, stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) a.dist[i] = a.inf;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < a.V; v += stride) a.stamp[v] = ~0u;
}

// Sources: label 0 in their lane; each distinct source once in the first
// frontier.
__global__ void ms_sources_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    if (threadIdx.x != 0) return;
    uint32_t n = 0;
    for (uint32_t l = 0; l < a.k; ++l) {
        const uint32_t s = a.sources[l];
        a.dist[size_t(s) * kML + l] = 0u;
        bool seen = false;
        for (uint32_t j = 0; j < l; ++j) seen |= a.sources[j] == s;
        if (!seen) {
            a.queue[0][n++] = s;
            a.stamp[s] = 0u;
            a.hdr->frontier_edges += a.row_off[s + 1] - a.row_off[s];  // round 0's frontier
        }
    }
    a.hdr->qsize[0] = n;
}


// Push round: a warp takes 32 frontier vertices; rows shorter than
// kHubDegree are walked as one combined edge list (each lane finds its
// edge's owner by a shuffle binary search and receives the owner's label
// row by shuffles), longer rows become hub tasks.
template <int WK>
__global__ void __launch_bounds__(kMSThreads) ms_expand_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || pull_round(a)) return;
    const View w = view(a);
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * kMSThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kMSThreads) >> 5;
    unsigned long long relaxed = 0;
    for (uint32_t base0 = gwarp * 32; base0 < w.qn; base0 += nwarps * 32) {
        const uint32_t i = base0 + lane;
        uint32_t deg = 0, u = 0;
        uint64_t off = 0;
        Row8 du;
#pragma unroll
        for (int l = 0; l < kML; ++l) du.d[l] = a.inf;
        if (i < w.qn) {
            u = w.q[i];
            off = a.row_off[u];
            const uint64_t full = a.row_off[u + 1] - off;
            relaxed += full;
            if (full >= kHubDegree) {
                const uint32_t nch = static_cast<uint32_t>((full + kHubChunk - 1) / kHubChunk);
                const uint32_t hb = atomicAdd(&a.hdr->hub_count, nch);
                for (uint32_t c = 0; c < nch; ++c) a.hubs[hb + c] = make_uint2(u, c);
            } else {
                deg = static_cast<uint32_t>(full);
                du = load_row(a.dist, u);
            }
        }
        uint32_t incl = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t b = 0; b < total; b += 32) {
            const uint32_t j = b + lane;
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1) {
                const uint32_t probe = __shfl_sync(0xffffffffu, incl, lo + step - 1);
                if (probe <= j) lo += step;
            }
            const uint32_t o_incl = __shfl_sync(0xffffffffu, incl, lo);
            const uint32_t o_deg = __shfl_sync(0xffffffffu, deg, lo);
            const uint64_t o_off = __shfl_sync(0xffffffffu, off, lo);
            Row8 ou;
#pragma unroll
            for (int l = 0; l < kML; ++l) ou.d[l] = __shfl_sync(0xffffffffu, du.d[l], lo);
            bool join = false;
            uint32_t v = 0;
            if (j < total) {
                const uint64_t e = o_off + (j - (o_incl - o_deg));
                v = dev::ld_stream(a.cols + e);
                join = relax_row<WK>(a, w, ou, v, ssc::edge_weight<WK>(a.weights, e));
            }
            const uint32_t vals[1] = {v};
            ssc::warp_append<1>(w.qnext, w.qnext_size, vals, join ? 1u : 0u, lane);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) relaxed += __shfl_xor_sync(0xffffffffu, relaxed, o);
    if (lane == 0 && relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
}

// One warp per kHubChunk-edge slice of a long frontier row.
template <int WK>
__global__ void __launch_bounds__(kMSThreads) ms_hub_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || pull_round(a)) return;
    const View w = view(a);
    const uint32_t n = *(volatile uint32_t *)&a.hdr->hub_count;
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * kMSThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kMSThreads) >> 5;
    for (uint32_t t = gwarp; t < n; t += nwarps) {
        const uint2 h = a.hubs[t];
        const uint64_t rb = a.row_off[h.x], re = a.row_off[h.x + 1];
        const uint64_t b = rb + uint64_t(h.y) * kHubChunk;
        const uint32_t len = static_cast<uint32_t>(((b + kHubChunk < re) ? b + kHubChunk : re) - b);
        const Row8 du = load_row(a.dist, h.x);
        for (uint32_t x = 0; x < len; x += 32) {
            bool join = false;
            uint32_t v = 0;
            if (x + lane < len) {
                const uint64_t e = b + x + lane;
                v = dev::ld_stream(a.cols + e);
                join = relax_row<WK>(a, w, du, v, ssc::edge_weight<WK>(a.weights, e));
            }
            const uint32_t vals[1] = {v};
            ssc::warp_append<1>(w.qnext, w.qnext_size, vals, join ? 1u : 0u, lane);
        }
    }
}

// Tile row r: lowers its labels to m where that improves them, with plain
// stores -- a tile row has exactly one writer during a sweep (the warp that
// owns its tile) and no push runs beside a sweep; true when r joins the
// next frontier.
__device__ __forceinline__ bool pull_store_row(const MSArgs &a, const View &w, uint32_t r, const Row8 &m) {
    const Row8 cur = load_row(a.dist, r);
    Row8 nx;
    bool improved = false;
#pragma unroll
    for (int l = 0; l < kML; ++l) {
        const bool lower = l < static_cast<int>(a.k) && m.d[l] < cur.d[l];
        nx.d[l] = lower ? m.d[l] : cur.d[l];
        improved |= lower;
    }
    if (!improved) return false;
    uint4 *p = reinterpret_cast<uint4 *>(a.dist + size_t(r) * kML);
    p[0] = make_uint4(nx.d[0], nx.d[1], nx.d[2], nx.d[3]);
    p[1] = make_uint4(nx.d[4], nx.d[5], nx.d[6], nx.d[7]);
    a.stamp[r] = w.next_stamp;
    return true;
}

// Lowers row r's labels to m (lanes that improve); true when r joins the
// next frontier now.  Long rows: every chunk of the row may lower it.
__device__ __forceinline__ bool pull_lower(const MSArgs &a, const View &w, uint32_t r, const Row8 &m) {
    const Row8 cur = load_row(a.dist, r);
    bool improved = false;
#pragma unroll
    for (int l = 0; l < kML; ++l)
        if (l < static_cast<int>(a.k) && m.d[l] < cur.d[l])
            improved |= m.d[l] < atomicMin(a.dist + size_t(r) * kML + l, m.d[l]);
    return improved && atomicExch(a.stamp + r, w.next_stamp) != w.next_stamp;
}

// Per-lane minimum of d[u] + w over in-edges [lo, hi) into m (ids at
// slot[x - a0]: staged, or the CSC itself); each thread of the caller walks
// its own edges lo, lo + step, ..., kPullU of them loaded before any is
// relaxed so that their label-row gathers overlap.  Labels are read live
// (not snapshotted): rows lowered earlier in the same sweep -- the hub rows,
// whose chunks come first -- feed the rows after them.
constexpr int kPullU = 4;

template <int WK>
__device__ __forceinline__ void pull_edges(const MSArgs &a, const uint32_t *s_hot, const uint32_t *slot, uint64_t a0,
                                           uint64_t lo, uint64_t hi, uint64_t step, uint64_t pol, Row8 &m) {
    for (uint64_t x0 = lo; x0 < hi; x0 += step * kPullU) {
        uint32_t u[kPullU], wt[kPullU];
#pragma unroll
        for (int j = 0; j < kPullU; ++j) {
            const uint64_t x = x0 + j * step;
            u[j] = x < hi ? slot[x - a0] : 0u;
            wt[j] = x < hi ? ssc::edge_weight<WK>(a.in_w, x) : 0u;
        }
#pragma unroll
        for (int j = 0; j < kPullU; ++j)
            if (u[j] & kHotTag) u[j] = s_hot[u[j] & ~kHotTag];
        Row8 du[kPullU];
#pragma unroll
        for (int j = 0; j < kPullU; ++j) {
            if (x0 + j * step < hi) {
                du[j] = load_row_keep(a.dist, u[j], pol);
            } else {
#pragma unroll
                for (int l = 0; l < kML; ++l) du[j].d[l] = a.inf;
            }
        }
#pragma unroll
        for (int j = 0; j < kPullU; ++j)
#pragma unroll
            for (int l = 0; l < kML; ++l)
                if (du[j].d[l] != a.inf) m.d[l] = min(m.d[l], extend<WK>(du[j].d[l], wt[j]));
    }
}

// kStaged: ids staged into shared memory by bulk copies (tiles fit a
// staging slot); otherwise read from global memory in place.
template <int WK, bool kStaged>
__global__ void __launch_bounds__(kMPThreads, 1) ms_pull_kernel(const MSArgs *__restrict__ args) {
    extern __shared__ __align__(128) unsigned char s_stage[];
    const MSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || !pull_round(a)) return;
    const View w = view(a);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    stage::WarpStage ws{};
    if constexpr (kStaged) ws = stage::warp_stage(s_stage, warp, lane);
    uint32_t *s_hot = reinterpret_cast<uint32_t *>(s_stage + (kStaged ? stage::kStageBytes : 0));
    for (uint32_t i = threadIdx.x; i < a.num_hot; i += blockDim.x) s_hot[i] = a.hot_vertex[i];
    __syncthreads();
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t nwarps = uint64_t(gridDim.x) * (kMPThreads / 32);
    const uint64_t first = uint64_t(blockIdx.x) * (kMPThreads / 32) + warp;
    Row8 acc;  // per-lane minima of the current chunk
    auto task = [&](uint4 d, uint64_t, uint32_t j, uint32_t nu, const uint32_t *slot, uint64_t a0) {
            if (task_is_chunk(d)) {
                const stage::Unit u = stage::unit_of(d, j);
                if (j == 0)
#pragma unroll
                    for (int l = 0; l < kML; ++l) acc.d[l] = a.inf;
                pull_edges<WK>(a, s_hot, slot, a0, u.lo + lane, u.hi, 32, pol, acc);
                if (j + 1 < nu) return;
                Row8 m = acc;
#pragma unroll
                for (int l = 0; l < kML; ++l)
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) m.d[l] = min(m.d[l], __shfl_xor_sync(0xffffffffu, m.d[l], o));
                if (lane == 0) {
                    const uint32_t row = a.long_rows[d.z].row;
                    if (pull_lower(a, w, row, m)) ssc::append(w.qnext, w.qnext_size, row);
                }
                return;
            }
            // tile: rows [r0, rl); short rows one lane each, rows of >= 64
            // in-edges by the whole warp
            const uint32_t r0 = d.z, rl = d.w;
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t rr = rb + lane;
                const bool active = rr < rl;
                const uint64_t lo = active ? a.in_off[rr] : 0, hi = active ? a.in_off[rr + 1] : 0;
                bool joined = false;
                if (active && hi - lo < 64) {
                    Row8 m;
#pragma unroll
                    for (int l = 0; l < kML; ++l) m.d[l] = a.inf;
                    pull_edges<WK>(a, s_hot, slot, a0, lo, hi, 1, pol, m);
                    joined = pull_store_row(a, w, rr, m);
                }
                uint32_t big = __ballot_sync(0xffffffffu, active && (hi - lo >= 64));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, hi, src);
                    Row8 m;
#pragma unroll
                    for (int l = 0; l < kML; ++l) m.d[l] = a.inf;
                    pull_edges<WK>(a, s_hot, slot, a0, bb + lane, ee, 32, pol, m);
#pragma unroll
                    for (int l = 0; l < kML; ++l)
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1)
                            m.d[l] = min(m.d[l], __shfl_xor_sync(0xffffffffu, m.d[l], o));
                    const bool jn = (lane == 0) && pull_store_row(a, w, rb + src, m);
                    if (__shfl_sync(0xffffffffu, jn ? 1u : 0u, 0) && lane == src) joined = true;
                }
                const uint32_t vals[1] = {rr};
                ssc::warp_append<1>(w.qnext, w.qnext_size, vals, joined ? 1u : 0u, lane);
            }
        };
    bool ok = true;
    if constexpr (kStaged)
        ok = stage::stage_pipeline(a.tasks, a.in_src, first, nwarps, a.num_tasks, ws, lane, task);
    else
        stage::direct_tasks(a.tasks, a.in_src, first, nwarps, a.num_tasks, task);
    if (!ok) {
        atomicExch(&a.hdr->error, 1u);
        atomicExch(&a.hdr->done, 1u);
        if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&a.hdr->relaxations, static_cast<unsigned long long>(a.num_edges));
        atomicAdd(&a.hdr->pull_rounds, 1u);
    }
}

// Round-end bookkeeping (one thread): true when the solve is finished.
__device__ __forceinline__ bool ms_end_round(const MSArgs &a, MSHeader *h) {
    const uint32_t r = h->round;
    const uint32_t n_next = h->qsize[(r + 1) & 1];
    h->frontier_total += h->qsize[r & 1];
    h->qsize[r & 1] = 0;
    h->hub_count = 0;
    h->frontier_edges = 0;
    h->round = r + 1;
    const bool conv = n_next == 0;
    if (conv || r + 1 >= h->max_rounds) {
        h->done = 1;
        h->converged = conv ? 1u : 0u;
        if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
        return true;
    }
    return false;
}

__global__ void ms_round_end_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    MSHeader *h = a.hdr;
    if (h->done) return;
    ms_end_round(a, h);
}

// End of a round of a pull-capable solve, in one grid launch: the whole
// grid sums the out-edges of the next frontier (the next round's push /
// pull decision), then the last block to finish ends the round.
__global__ void __launch_bounds__(kMSThreads) ms_round_close_kernel(const MSArgs *__restrict__ args) {
    const MSArgs a = *args;
    MSHeader *h = a.hdr;
    if (*(volatile uint32_t *)&h->done) return;
    const uint32_t r = *(volatile uint32_t *)&h->round;
    const uint32_t qn = *(volatile uint32_t *)&h->qsize[(r + 1) & 1];
    const uint32_t *q = ((r + 1) & 1) ? a.queue[1] : a.queue[0];
    unsigned long long sum = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < qn; i += gridDim.x * blockDim.x) {
        const uint32_t v = q[i];
        sum += a.row_off[v + 1] - a.row_off[v];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&h->frontier_edges_next, sum);
    __shared__ uint32_t s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&h->close_ticket, 1u) == gridDim.x - 1 ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    const unsigned long long fe = atomicAdd(&h->frontier_edges_next, 0ull);
    h->frontier_edges_next = 0;
    h->close_ticket = 0;
    ms_end_round(a, h);
    h->frontier_edges = fe;
}

// out[l][c] = dist[inv[c]][l] (caller order c; inv NULL: identity).
__global__ void ms_emit_kernel(const uint32_t *__restrict__ dist, const uint32_t *__restrict__ inv, uint64_t V,
                               uint32_t k, uint32_t *__restrict__ out) {
    for (uint64_t c = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; c < V; c += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = inv ? inv[c] : static_cast<uint32_t>(c);
        const Row8 r = load_row(dist, v);
        for (uint32_t l = 0; l < k; ++l) out[l * V + c] = r.d[l];
    }
}

template <int WK>
int ms_push_grid() {
    static int g = 0;
    if (g == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_expand_kernel<WK>, kMSThreads, 0));
        g = sm_count() * std::max(per_sm, 1);
    }
    return g;
}

template <int WK>
void ms_solve(GraphImpl &g, const uint32_t *sources, uint32_t k, uint32_t max_rounds, uint32_t flags, cudaStream_t s,
              uint32_t *out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    if (g.ms_dist.count < V * kML) g.ms_dist.allocate(V * kML);
    if (g.stamp.count < 2 * V) g.stamp.allocate(2 * V);
    for (int i = 0; i < 2; ++i)
        if (g.queue[i].count < V) g.queue[i].allocate(V);
    const uint64_t hub_cap = V + g.E / kHubChunk + 2;
    if (g.hub_tasks.count < hub_cap) g.hub_tasks.allocate(hub_cap);
    const size_t sb = 512 + sizeof(MSHeader);
    if (g.ms_state.count < sb) g.ms_state.allocate(sb);
    MSArgs *d_args = reinterpret_cast<MSArgs *>(g.ms_state.get());
    MSHeader *hdr = reinterpret_cast<MSHeader *>(g.ms_state.get() + 256);
    static_assert(sizeof(MSArgs) <= 256, "MSArgs must fit its 256-byte slot");

    MSArgs a{};
    a.row_off = g.row_offsets.get();
    a.cols = g.cols.get();
    a.weights = g.weights.get();
    a.dist = g.ms_dist.get();
    a.stamp = g.stamp.get();
    a.queue[0] = g.queue[0].get();
    a.queue[1] = g.queue[1].get();
    a.hubs = g.hub_tasks.get();
    a.hdr = hdr;
    a.V = static_cast<uint32_t>(V);
    a.k = k;
    a.inf = (WK == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
    a.num_edges = g.E;
    for (uint32_t l = 0; l < k; ++l) a.sources[l] = graph_vertex(g, sources[l], s);
    // staged pull when the graph's tiles fit a staging slot, else ids read in place
    const bool staged = g.tile_cost <= kStageTileMax && stage::staged_shared_bytes(g.num_hot) <= kPRSmemMax;
    const bool pull_ok = (g.flags & HYT_GRAPH_PULL) && (WK == HYT_WEIGHTS_NONE || g.in_weights.get()) && g.E > 0 &&
                         g.pull_tasks.get() && size_t(g.num_hot) * 4 <= kPRSmemMax;
    a.pull_div = pull_ok ? 4u : 0u;
    if (pull_ok) {
        a.in_off = g.in_offsets.get();
        a.in_src = g.in_sources.get();
        a.in_w = g.in_weights.get();
        a.hot_vertex = g.hot_vertex.get();
        a.long_rows = g.long_rows.get();
        a.tasks = g.pull_tasks.get();
        a.num_tasks = g.num_chunks + g.num_tiles;
        a.num_hot = g.num_hot;
    }
    const unsigned pull_smem =
        static_cast<unsigned>(staged ? stage::staged_shared_bytes(g.num_hot) : size_t(g.num_hot) * 4);
    const void *pull_fn = staged ? reinterpret_cast<const void *>(ms_pull_kernel<WK, true>)
                                 : reinterpret_cast<const void *>(ms_pull_kernel<WK, false>);
    static bool attr = false;
    if (!attr) {
        HYT_CUDA(cudaFuncSetAttribute(ms_pull_kernel<WK, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaFuncSetAttribute(ms_pull_kernel<WK, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        attr = true;
    }
    const int grid = ms_push_grid<WK>();
    const int pgrid = sm_count();

    MSHeader h0{};
    h0.max_rounds = max_rounds;
    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        HYT_CUDA(cudaGraphCreate(&graph, 0));
        HYT_CUDA(cudaGraphConditionalHandleCreate(&a.cond, graph, 1, cudaGraphCondAssignDefault));
        a.use_cond = 1;
    }
    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaMemcpyAsync(hdr, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    ms_init_kernel<<<grid_for(V * kML, 256, 148 * 8), 256, 0, s>>>(d_args);
    ms_sources_kernel<<<1, 32, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 2;
    if (use_graph) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = a.cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        HYT_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        void *kargs[] = {&d_args};
        cudaGraphNode_t prev = nullptr, node;
        auto add = [&](const void *f, dim3 gd, dim3 bd, unsigned smem) {
            cudaKernelNodeParams kp = {};
            kp.func = const_cast<void *>(f);
            kp.gridDim = gd;
            kp.blockDim = bd;
            kp.sharedMemBytes = smem;
            kp.kernelParams = kargs;
            HYT_CUDA(cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
            prev = node;
        };
        add(reinterpret_cast<void *>(ms_expand_kernel<WK>), dim3(grid), dim3(kMSThreads), 0);
        add(reinterpret_cast<void *>(ms_hub_kernel<WK>), dim3(grid), dim3(kMSThreads), 0);
        if (a.pull_div) {
            add(pull_fn, dim3(pgrid), dim3(kMPThreads), pull_smem);
            add(reinterpret_cast<void *>(ms_round_close_kernel), dim3(grid), dim3(kMSThreads), 0);
        } else {
            add(reinterpret_cast<void *>(ms_round_end_kernel), dim3(1), dim3(1), 0);
        }
        HYT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        HYT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        for (uint32_t r = 0; r < max_rounds; ++r) {
            ms_expand_kernel<WK><<<grid, kMSThreads, 0, s>>>(d_args);
            ms_hub_kernel<WK><<<grid, kMSThreads, 0, s>>>(d_args);
            if (a.pull_div) {
                void *pargs[] = {&d_args};
                HYT_CUDA(cudaLaunchKernel(pull_fn, dim3(pgrid), dim3(kMPThreads), pargs, pull_smem, s));
            }
            if (a.pull_div)
                ms_round_close_kernel<<<grid, kMSThreads, 0, s>>>(d_args);
            else
                ms_round_end_kernel<<<1, 1, 0, s>>>(d_args);
            HYT_CUDA(cudaGetLastError());
            launches += a.pull_div ? 4 : 3;
            uint32_t done = 0;
            HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            if (done) break;
        }
    }
    MSHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (use_graph) launches += (a.pull_div ? 4 : 3) * h.round;
    if (h.error) fail(HYT_E_TIMEOUT, "hyt_sssp_multi: a bounded wait for a staged copy ran out");
    if (out) {
        if (is_device_pointer(out)) {
            ms_emit_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.ms_dist.get(), g.inv.get(), V, k, out);
            HYT_CUDA(cudaGetLastError());
        } else {
            Scratch<uint32_t> tmp(V * k, s);
            ms_emit_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.ms_dist.get(), g.inv.get(), V, k, tmp.get());
            HYT_CUDA(cudaGetLastError());
            copy_from_device(out, tmp.get(), V * k * sizeof(uint32_t), s);
        }
    }
    HYT_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->iterations = h.round;
        stats->converged = h.converged;
        stats->device_ms = total_ms;
        stats->total_launches = launches;
        stats->edges_processed = h.relaxations;
        stats->vertices_processed = h.frontier_total;
        // per frontier vertex: 8 B offset pair (read twice) + 32 B label row
        // + 4 B queue entry; per relaxed edge: 4 B column + 4 B weight + a
        // 32 B label row
        stats->algorithmic_bytes = 52ull * h.frontier_total + 40ull * h.relaxations;
    }
}

}  // namespace

void sssp_multi(GraphImpl &g, const uint32_t *sources, uint32_t k, uint32_t max_rounds, uint32_t flags,
                cudaStream_t s, uint32_t *out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PUSH");
    if (!sources) fail(HYT_E_INVALID, "sources is NULL");
    if (k == 0 || k > kML) fail(HYT_E_INVALID, "hyt_sssp_multi takes 1 to 8 sources");
    for (uint32_t l = 0; l < k; ++l)
        if (sources[l] >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
    const uint64_t cap = std::min<uint64_t>(4 * g.V + 1024, 0x7FFFFFFFull);
    const uint32_t rounds = max_rounds ? max_rounds : static_cast<uint32_t>(cap);
    switch (g.weight_kind) {
        case HYT_WEIGHTS_NONE: ms_solve<HYT_WEIGHTS_NONE>(g, sources, k, rounds, flags, s, out, stats); break;
        case HYT_WEIGHTS_U32: ms_solve<HYT_WEIGHTS_U32>(g, sources, k, rounds, flags, s, out, stats); break;
        case HYT_WEIGHTS_F32: ms_solve<HYT_WEIGHTS_F32>(g, sources, k, rounds, flags, s, out, stats); break;
        default: fail(HYT_E_INTERNAL, "unknown weight kind");
    }
}

}  // namespace hyt
