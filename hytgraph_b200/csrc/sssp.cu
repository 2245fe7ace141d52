// Single-source shortest paths: frontier push over the CSR with atomicMin.
//
// The reference solver (src/algorithms/sssp.cpp:109-234, cuda/sssp.cu:
// 100-154) is a synchronous Bellman-Ford that pulls over all in-edges every
// round.  Any label-correcting schedule reaches the same fixed point
//     d[s] = 0,  d[v] = min_{u->v} (d[u] + w(u,v))
// because every relaxation only lowers a label to a value that some path
// attains; so distances are bit-identical to the reference.  Integer (u32)
// weights relax with exact integer adds; float weights relax with the same
// IEEE add the reference uses, compared as ordered bit patterns (valid for
// non-negative floats).
//
// Schedule: near/far buckets (Delta-stepping with one far pile).  Vertices
// whose label drops below the current threshold T join the next near
// frontier; the others go to the far pile.  When the near frontier runs
// dry, T grows by Delta and the far pile is split: entries now below T
// become the near frontier, entries below the old threshold are stale
// (already settled) and are dropped.  Delta = infinity is plain frontier
// Bellman-Ford (used for float weights).
//
// Expansion is warp-centric: a warp takes 32 frontier vertices, prefix-sums
// their degrees with shuffles and walks the combined edge list 32 edges at
// a time, finding each edge's owner with a 5-step shuffle binary search.
// Rows of >= kHubDegree edges become kHubChunk-edge warp tasks for a second
// grid-wide kernel, so no warp owns more than ~2K edges of a round.  Each
// lane keeps 4 edges in flight through loads and atomics (relax_batch).  A
// vertex joins a frontier once per round (round stamp) and the far pile once
// per phase (phase stamp), appended with one warp-aggregated atomic.
//
// With one bucket and a CSC, a round whose frontier carries more than
// E / pull_div out-edges runs as a pull sweep over the CSC instead
// (sssp_pull_kernel: 512-unit tiles, labels gathered 8 per lane in flight,
// tile rows written with plain stores).  A sweep skips the rows whose label
// is at most (lowest frontier label + smallest weight): no in-edge can
// lower them, so their in-edges are neither read nor gathered (the round
// close finds the frontier's lowest label).  All round state lives on the
// device; inside a CUDA graph the rounds run as a conditional while-loop
// (expand, hub chunks, pull sweep, round close), instantiated once per
// graph and launched again by later solves.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>

#include "common.cuh"
#include "graph.cuh"
#include "host_checks.hpp"
#include "scratch.cuh"
#include "hybrid.cuh"
#include "solvers.cuh"
#include "sssp_core.cuh"
#include "stage.cuh"

namespace hyt {
namespace {

using namespace ssc;

// Splits the far pile at the start of a round whose near frontier is empty.
__global__ void __launch_bounds__(kSSThreads) sssp_split_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    const SSHeader *h = a.hdr;
    if (*(volatile const uint32_t *)&h->done || !*(volatile const uint32_t *)&h->pending) return;
    const uint32_t n = (h->phase & 1) ? h->fsize[1] : h->fsize[0];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) split_entry(a, i);
}

// HYB: the edges of a vertex's partition are reached through a.loc
// (partitioned solves); compacted partitions are expanded from their packed
// payload by sssp_expand_packed_kernel instead.
template <int WK, bool HYB = false>
__global__ void __launch_bounds__(kSSThreads) sssp_expand_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || pull_round(a)) return;
    const RoundView rv = round_view(a);
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * kSSThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kSSThreads) >> 5;
    unsigned long long relaxed = 0, improved = 0;
    auto hub = [&](uint32_t v, uint32_t nch) {
        const uint32_t base = atomicAdd(&a.hdr->hub_count, nch);
        for (uint32_t c = 0; c < nch; ++c) a.hubs[base + c] = make_uint2(v, c);
    };
    for (uint32_t w = gwarp; uint64_t(w) * 32 < rv.qn; w += nwarps)
        expand_warp<WK, HYB, HYB ? kEdgeBatch : 16>(a, rv, w * 32, lane, kHubDegree, relaxed, improved, hub);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) relaxed += __shfl_xor_sync(0xffffffffu, relaxed, o);
    if (lane == 0 && relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
}

// One warp per kHubChunk-edge slice of a long frontier row.
template <int WK, bool HYB = false>
__global__ void __launch_bounds__(kSSThreads) sssp_hub_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || pull_round(a)) return;
    const RoundView rv = round_view(a);
    const uint32_t n = *(volatile uint32_t *)&a.hdr->hub_count;
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * kSSThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kSSThreads) >> 5;
    unsigned long long improved = 0;
    for (uint32_t t = gwarp; t < n; t += nwarps) {
        const uint2 h = a.hubs[t];
        const uint32_t *hc = a.cols, *hw = a.weights;
        if constexpr (HYB) {
            const EdgeLoc L = a.loc[h.x >> a.part_shift];
            hc = L.cols;
            hw = L.weights;
        }
        hub_chunk<WK>(a, rv, hc, hw, h.x, h.y, lane, improved);
    }
}

// ---- pull sweeps (direction-optimised rounds) ------------------------------
//
// A round whose frontier carries more than E / pull_div out-edges is run as
// a sweep over the CSC instead: every vertex takes the minimum of
// d[u] + w(u, v) over its in-edges (no atomics on the edge path, streaming
// reads of ids and weights, label gathers from L2), and improved vertices
// form the next frontier.  Any label-correcting schedule reaches the same
// fixed point, so distances are unchanged.  Single-bucket solves only.

// CSC of the graph for pull sweeps (PageRank's tiles and long-row chunks).
struct PullGraph {
    const uint64_t *in_off;
    const uint32_t *in_src;   // hot sources tagged kHotTag | slot
    const uint32_t *in_w;     // weights in CSC order (NULL when unweighted)
    const uint32_t *tile_start;
    const LongRow *long_rows;
    const uint2 *chunk_tasks;
    const uint32_t *hot_vertex;
    const uint4 *tasks;       // pull task descriptors (next-task prefetch, staged sweeps)
    uint64_t num_tiles, num_chunks;
    uint32_t tile_cost;
    uint32_t num_hot;
};


// Lowers tile row r's label from `seen` to c if that improves it; true when
// r joins the next frontier.  A tile row has exactly one writer during a
// sweep (the warp that owns its tile) and no push runs beside a sweep, so
// `seen` -- read before the tile's gathers -- is the row's label, and plain
// stores replace the atomics.
__device__ __forceinline__ bool pull_store(const SSArgs &a, const RoundView &rv, uint32_t r, uint32_t c,
                                           uint32_t seen) {
    if (c >= seen) return false;
    a.dist[r] = c;
    a.stamp[r] = rv.next_stamp;
    return true;
}

// Lowers row r's label to c if that improves it; returns true when r joins
// the next frontier for the first time this round.
__device__ __forceinline__ bool pull_relax(const SSArgs &a, const RoundView &rv, uint32_t r, uint32_t c) {
    if (c >= __ldcg(a.dist + r)) return false;
    const uint32_t old = atomicMin(a.dist + r, c);
    if (c >= old) return false;
    return atomicExch(a.stamp + r, rv.next_stamp) != rv.next_stamp;
}

// Candidate labels d[u] + w of in-edges [lo, hi), kPullBatch per lane in
// flight: all ids and weights, hot slots mapped to vertex ids through the
// CTA's shared-memory table, all labels gathered evict-last from L2, then
// the sink.  Unreached sources give infinity.
#ifndef HYT_PULL_BATCH
#define HYT_PULL_BATCH 8  // 16: register spills and 5 % slower sweeps at R-MAT scale 24
#endif
constexpr int kPullBatch = HYT_PULL_BATCH;

// One pass of kK batches (edges lo + base + 32k + lane, k < kK).  With
// kMask, edges whose bit is set in `skip` (bit i of word i / 32) belong to
// skipped rows: they are neither read nor gathered.
template <int kK, int WK, bool kMask, class Sink>
__device__ __forceinline__ void pull_pass(const SSArgs &a, const PullGraph &pg, const uint32_t *s_hot, uint64_t lo,
                                          uint32_t base, uint32_t n, uint64_t pol, int lane, const uint32_t *skip,
                                          Sink &sink) {
    // ids, then the label gathers, then the weights (streamed; issued after
    // the gathers so that ids and weights are not live together)
    uint32_t id[kK], w[kK], du[kK];
    bool live[kK];
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const uint32_t i = base + 32 * k + lane;
        live[k] = i < n && !(kMask && ((skip[(base >> 5) + k] >> lane) & 1u));
        id[k] = live[k] ? dev::ld_stream(pg.in_src + lo + i) : 0u;
    }
#pragma unroll
    for (int k = 0; k < kK; ++k)
        if (id[k] & kHotTag) id[k] = s_hot[id[k] & ~kHotTag];  // hot slot -> vertex id
#pragma unroll
    for (int k = 0; k < kK; ++k) du[k] = (!kMask || live[k]) ? dev::ld_keep_u32(a.dist + id[k], pol) : a.inf;
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const uint32_t i = base + 32 * k + lane;
        w[k] = live[k] ? edge_weight<WK>(pg.in_w, lo + i) : 0u;
    }
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const uint32_t i = base + 32 * k + lane;
        if (live[k]) sink(i, du[k] == a.inf ? a.inf : extend<WK>(du[k], w[k]));
    }
}

// The last, partial pass issues only the 4-batch groups that hold edges
// (a warp-uniform choice); the edges and their order are the same.
template <int WK, bool kMask, class Sink>
__device__ __forceinline__ void pull_span(const SSArgs &a, const PullGraph &pg, const uint32_t *s_hot, uint64_t lo,
                                          uint64_t hi, uint64_t pol, int lane, const uint32_t *skip, Sink &&sink) {
    static_assert(kPullBatch % 4 == 0 && kPullBatch >= 4, "batches come in groups of 4");
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    for (uint32_t base = 0; base < n; base += 32 * kPullBatch) {
        const uint32_t groups = (n - base + 127) / 128;
        if (groups >= kPullBatch / 4)
            pull_pass<kPullBatch, WK, kMask>(a, pg, s_hot, lo, base, n, pol, lane, skip, sink);
        else if (groups == 1)
            pull_pass<4, WK, kMask>(a, pg, s_hot, lo, base, n, pol, lane, skip, sink);
        else if (groups == 2)
            pull_pass<8, WK, kMask>(a, pg, s_hot, lo, base, n, pol, lane, skip, sink);
        else
            pull_pass<(kPullBatch >= 12 ? 12 : kPullBatch), WK, kMask>(a, pg, s_hot, lo, base, n, pol, lane, skip, sink);
    }
}

#ifndef HYT_PULL_THREADS
#define HYT_PULL_THREADS 1024
#endif
constexpr int kPullThreads = HYT_PULL_THREADS;  // one CTA per SM, like the PageRank kernel

// Row skipping.  Let F be this round's frontier (every vertex whose label
// dropped since its out-edges were last relaxed) and fmin its lowest label.
// An in-edge (u, v) can lower d[v] this round only if u is in F, and then
// its candidate is d[u] + w >= fmin + min_w.  So a row with
// d[v] <= extend(fmin, min_w) cannot improve: its in-edges are neither
// read nor gathered.  A vertex lowered during the round joins the next
// frontier, so the argument holds again next round; distances are
// unchanged.
template <int WK>
__device__ __forceinline__ uint32_t skip_bound(const SSArgs &a, bool &on) {
    const uint32_t fmin = *(volatile const uint32_t *)&a.hdr->fmin;
    on = a.skip_rows && fmin < a.inf;
    return on ? extend<WK>(fmin, a.min_w) : 0u;
}

// Sets bits [lo, hi) of a warp's edge mask (shared-memory words).
__device__ __forceinline__ void mask_range(uint32_t *mw, uint32_t lo, uint32_t hi) {
    for (uint32_t x = lo; x < hi;) {
        const uint32_t b = x & 31, cnt = min(32u - b, hi - x);
        atomicOr(mw + (x >> 5), (cnt == 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u)) << b);
        x += cnt;
    }
}

template <int WK>
__global__ void __launch_bounds__(kPullThreads, 1) sssp_pull_kernel(const SSArgs *__restrict__ args, PullGraph pg) {
    extern __shared__ __align__(16) uint32_t s_dyn_u[];
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || !pull_round(a)) return;
    const RoundView rv = round_view(a);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // vertex ids of the hot slots (tagged sources in the CSC)
    uint32_t *s_hot = s_dyn_u;
    for (uint32_t i = threadIdx.x; i < pg.num_hot; i += blockDim.x) s_hot[i] = pg.hot_vertex[i];
    __syncthreads();
    uint32_t *sv = s_dyn_u + pg.num_hot + warp * (2 * pg.tile_cost + 8);
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t total = pg.num_chunks + pg.num_tiles;
    const uint64_t nwarps = uint64_t(gridDim.x) * (kPullThreads / 32);
    const uint32_t *pf_w = (WK == HYT_WEIGHTS_NONE) ? nullptr : pg.in_w;
    bool skip_on;
    const uint32_t skip_at = skip_bound<WK>(a, skip_on);
    unsigned long long relaxed = 0;  // in-edges this lane's warp relaxed (lane 0 counts tiles and chunks)
    for (uint64_t task = uint64_t(blockIdx.x) * (kPullThreads / 32) + warp; task < total; task += nwarps) {
        // the next task's descriptor now; its edge lines are warmed in L2
        // once this task's gathers are issued
        const uint64_t next = task + nwarps;
        const uint4 nd = next < total ? pg.tasks[next] : make_uint4(0, 0, 0, 0);
        if (task < pg.num_chunks) {
            // slice of a long row: warp minimum, then one relaxation
            const uint2 t = pg.chunk_tasks[task];
            const LongRow L = pg.long_rows[t.x];
            const uint64_t rb = pg.in_off[L.row], re = pg.in_off[L.row + 1];
            const uint64_t lo = rb + uint64_t(t.y) * kLongChunk;
            const uint64_t hi = (lo + kLongChunk < re) ? lo + kLongChunk : re;
            if (skip_on && __shfl_sync(0xffffffffu, __ldcg(a.dist + L.row), 0) <= skip_at) continue;
            if (lane == 0) relaxed += hi - lo;
            uint32_t best = a.inf;
            pull_span<WK, false>(a, pg, s_hot, lo, hi, pol, lane, nullptr,
                                 [&](uint32_t, uint32_t c) { best = min(best, c); });
            prefetch_task(nd, pg.in_src, pf_w, lane);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (lane == 0 && pull_relax(a, rv, L.row, best)) append(rv.qnext, rv.qnext_size, L.row);
        } else {
            // merge-path tile of short rows: candidates staged per edge
            const uint64_t k = task - pg.num_chunks;
            const uint32_t r0 = pg.tile_start[k], r1 = pg.tile_start[k + 1];
            if (r0 == r1) continue;
            const uint64_t last_b = pg.in_off[r1 - 1], last_e = pg.in_off[r1];
            const uint32_t rl = (last_e - last_b >= pg.tile_cost) ? r1 - 1 : r1;  // long last row is chunked
            const uint64_t e0 = pg.in_off[r0];
            const uint64_t e1 = (rl == r1) ? last_e : last_b;
            // the first 32 rows' bounds (relative to e0) and labels, loaded
            // before the gathers so that they arrive with them
            uint32_t lo_p = 0, hi_p = 0, seen_p = 0;
            if (r0 + lane < rl) {
                lo_p = static_cast<uint32_t>(pg.in_off[r0 + lane] - e0);
                hi_p = static_cast<uint32_t>(pg.in_off[r0 + lane + 1] - e0);
                seen_p = __ldcg(a.dist + r0 + lane);
            }
            if (lane == 0) relaxed += e1 - e0;
            // rows that cannot improve: their edges' bits in a mask kept at
            // the end of the warp's slice, past the tile's candidates (no
            // shared memory beyond the slice: more would shrink L1)
            const uint32_t *skip = nullptr;
            const uint32_t words = static_cast<uint32_t>((e1 - e0 + 31) >> 5);
            if (skip_on && (e1 - e0) + words <= 2 * pg.tile_cost + 8) {
                uint32_t *mw = sv + (2 * pg.tile_cost + 8) - words;
                for (uint32_t x = lane; x < words; x += 32) mw[x] = 0u;
                __syncwarp();
                uint32_t any = 0;
                for (uint32_t rb = r0; rb < rl; rb += 32) {
                    const uint32_t r = rb + lane;
                    uint32_t lo = lo_p, hi = hi_p, seen = seen_p;
                    if (rb != r0 && r < rl) {
                        lo = static_cast<uint32_t>(pg.in_off[r] - e0);
                        hi = static_cast<uint32_t>(pg.in_off[r + 1] - e0);
                        seen = __ldcg(a.dist + r);
                    }
                    const bool sk = r < rl && seen <= skip_at;
                    any |= __ballot_sync(0xffffffffu, sk);
                    if (sk) {
                        relaxed -= hi - lo;
                        mask_range(mw, lo, hi);
                    }
                }
                __syncwarp();
                if (any) skip = mw;
            }
            if (skip)
                pull_span<WK, true>(a, pg, s_hot, e0, e1, pol, lane, skip, [&](uint32_t i, uint32_t c) { sv[i] = c; });
            else
                pull_span<WK, false>(a, pg, s_hot, e0, e1, pol, lane, nullptr,
                                     [&](uint32_t i, uint32_t c) { sv[i] = c; });
            prefetch_task(nd, pg.in_src, pf_w, lane);
            __syncwarp();
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t r = rb + lane;
                const bool active = r < rl;
                uint32_t lo = lo_p, hi = hi_p, seen = seen_p;
                if (rb != r0) {
                    lo = active ? static_cast<uint32_t>(pg.in_off[r] - e0) : 0u;
                    hi = active ? static_cast<uint32_t>(pg.in_off[r + 1] - e0) : 0u;
                    seen = active ? __ldcg(a.dist + r) : 0u;
                }
                bool joined = false;
                const bool live = active && !(skip && seen <= skip_at);  // skipped rows were not gathered
                if (live && hi - lo < 64) {
                    uint32_t best = a.inf;
                    for (uint32_t x = lo; x < hi; ++x) best = min(best, sv[x]);
                    joined = pull_store(a, rv, r, best, seen);
                }
                uint32_t big = __ballot_sync(0xffffffffu, live && (hi - lo >= 64));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint32_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint32_t ee = __shfl_sync(0xffffffffu, hi, src);
                    const uint32_t sn = __shfl_sync(0xffffffffu, seen, src);
                    uint32_t best = a.inf;
                    for (uint32_t x = bb + lane; x < ee; x += 32) best = min(best, sv[x]);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
                    const bool j = (lane == 0) && pull_store(a, rv, rb + src, best, sn);
                    if (__shfl_sync(0xffffffffu, j ? 1u : 0u, 0) && lane == src) joined = true;
                }
                const uint32_t vals[1] = {r};
                warp_append<1>(rv.qnext, rv.qnext_size, vals, joined ? 1u : 0u, lane);
            }
            __syncwarp();
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) relaxed += __shfl_xor_sync(0xffffffffu, relaxed, o);
    if (lane == 0 && relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.hdr->pull_rounds, 1u);
}

// ---- staged pull sweeps (CSC in HBM; pipeline in stage.cuh) ----------------

// Candidate labels d[u] + w of staged edges [lo, hi) (ids at slot[x - a0]):
// lane l takes edges lo + 32k + l; weights stream straight from HBM while
// the label gathers are in flight.  sink(i, candidate) receives edge lo + i.
template <int WK, class Sink>
__device__ __forceinline__ void pull_staged(const SSArgs &a, const PullGraph &pg, const uint32_t *s_hot,
                                            const uint32_t *slot, uint64_t a0, uint64_t lo, uint64_t hi, uint64_t pol,
                                            int lane, Sink &&sink) {
    constexpr int kB = stage::kUnitEdges / 32;
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    const uint32_t *ids = slot + (lo - a0);
    uint32_t w[kB], du[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const uint32_t i = 32 * k + lane;
        w[k] = (i < n) ? edge_weight<WK>(pg.in_w, lo + i) : 0u;
    }
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const uint32_t i = 32 * k + lane;
        uint32_t id = (i < n) ? ids[i] : 0u;
        if (id & kHotTag) id = s_hot[id & ~kHotTag];  // hot slot -> vertex id
        du[k] = dev::ld_keep_u32(a.dist + id, pol);
    }
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const uint32_t i = 32 * k + lane;
        if (i < n) sink(i, du[k] == a.inf ? a.inf : extend<WK>(du[k], w[k]));
    }
}

// pull_relax with the row's label read ahead of time: a stale (higher)
// label only lets through an atomicMin that then finds no improvement.
__device__ __forceinline__ bool pull_relax_seen(const SSArgs &a, const RoundView &rv, uint32_t r, uint32_t c,
                                                uint32_t seen) {
    if (c >= seen) return false;
    const uint32_t old = atomicMin(a.dist + r, c);
    if (c >= old) return false;
    return atomicExch(a.stamp + r, rv.next_stamp) != rv.next_stamp;
}

template <int WK>
__global__ void __launch_bounds__(stage::kStageThreads, 1) sssp_pull_staged_kernel(const SSArgs *__restrict__ args,
                                                                                   PullGraph pg) {
    extern __shared__ __align__(128) unsigned char s_stage[];
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done || !pull_round(a)) return;
    const RoundView rv = round_view(a);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const stage::WarpStage ws = stage::warp_stage(s_stage, warp, lane);
    uint32_t *s_hot = reinterpret_cast<uint32_t *>(s_stage + stage::kStageBytes);  // vertex ids of the hot slots
    for (uint32_t i = threadIdx.x; i < pg.num_hot; i += blockDim.x) s_hot[i] = pg.hot_vertex[i];
    __syncthreads();
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t total = pg.num_chunks + pg.num_tiles;
    const uint64_t nwarps = uint64_t(gridDim.x) * stage::kStageWarps;
    uint32_t best = a.inf;  // running minimum of the current chunk
    const bool ok = stage::stage_pipeline(
        pg.tasks, pg.in_src, uint64_t(blockIdx.x) * stage::kStageWarps + warp, nwarps, total, ws,
        lane, [&](uint4 d, uint64_t, uint32_t j, uint32_t nu, uint32_t *slot, uint64_t a0) {
            if (task_is_chunk(d)) {
                // slice of a long row: warp minimum, then one relaxation
                const stage::Unit u = stage::unit_of(d, j);
                if (j == 0) best = a.inf;
                pull_staged<WK>(a, pg, s_hot, slot, a0, u.lo, u.hi, pol, lane,
                                [&](uint32_t, uint32_t c) { best = min(best, c); });
                if (j + 1 < nu) return;
                uint32_t m = best;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
                if (lane == 0) {
                    const uint32_t row = pg.long_rows[d.z].row;
                    if (pull_relax(a, rv, row, m)) append(rv.qnext, rv.qnext_size, row);
                }
                return;
            }
            // merge-path tile of short rows: candidates replace the ids in
            // the slot, then each row takes its minimum
            const uint32_t r0 = d.z, rl = d.w;
            const uint64_t e0 = task_first_edge(d), e1 = e0 + task_edges(d);
            const uint32_t r = r0 + lane;
            const bool act0 = r < rl;
            const uint64_t lo0 = act0 ? pg.in_off[r] : 0, hi0 = act0 ? pg.in_off[r + 1] : 0;  // in flight
            const uint32_t seen0 = act0 ? __ldcg(a.dist + r) : 0u;
            pull_staged<WK>(a, pg, s_hot, slot, a0, e0, e1, pol, lane,
                            [&](uint32_t i, uint32_t c) { slot[e0 - a0 + i] = c; });
            __syncwarp();
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t rr = rb + lane;
                const bool active = rr < rl;
                const bool first = rb == r0;
                const uint64_t lo = first ? lo0 : (active ? pg.in_off[rr] : 0);
                const uint64_t hi = first ? hi0 : (active ? pg.in_off[rr + 1] : 0);
                bool joined = false;
                if (active && hi - lo < 64) {
                    uint32_t m = a.inf;
                    for (uint64_t x = lo; x < hi; ++x) m = min(m, slot[x - a0]);
                    joined = first ? pull_relax_seen(a, rv, rr, m, seen0) : pull_relax(a, rv, rr, m);
                }
                uint32_t big = __ballot_sync(0xffffffffu, active && (hi - lo >= 64));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, hi, src);
                    uint32_t m = a.inf;
                    for (uint64_t x = bb + lane; x < ee; x += 32) m = min(m, slot[x - a0]);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
                    const bool jn = (lane == 0) && pull_relax(a, rv, rb + src, m);
                    if (__shfl_sync(0xffffffffu, jn ? 1u : 0u, 0) && lane == src) joined = true;
                }
                const uint32_t vals[1] = {rr};
                warp_append<1>(rv.qnext, rv.qnext_size, vals, joined ? 1u : 0u, lane);
            }
        });
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

// End of a round of a pull-capable solve, in one grid launch: the whole
// grid sums the out-edges of the next frontier (the next round's push /
// pull decision) and, with row skipping, finds its lowest label; then the
// last block to finish runs the round-end logic.
__global__ void __launch_bounds__(kSSThreads) sssp_round_close_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    SSHeader *h = a.hdr;
    if (*(volatile uint32_t *)&h->done) return;
    const uint32_t r = *(volatile uint32_t *)&h->round;
    const uint32_t qn = *(volatile uint32_t *)&h->qsize[(r + 1) & 1];
    const uint32_t *q = ((r + 1) & 1) ? a.queue[1] : a.queue[0];
    unsigned long long sum = 0;
    uint32_t low = 0xFFFFFFFFu;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < qn; i += gridDim.x * blockDim.x) {
        const uint32_t v = q[i];
        sum += a.row_off[v + 1] - a.row_off[v];
        if (a.skip_rows) low = min(low, __ldcg(a.dist + v));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&h->frontier_edges_next, sum);
    if (a.skip_rows) {
        low = __reduce_min_sync(0xffffffffu, low);
        if ((threadIdx.x & 31) == 0 && low != 0xFFFFFFFFu) atomicMax(&h->fmin_inv, ~low);
    }
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
    h->fmin = ~atomicAdd(&h->fmin_inv, 0u);  // all ones when the next frontier is empty
    h->fmin_inv = 0;
    const bool finish = round_end(h);
    h->frontier_edges = fe;
    if (finish && a.use_cond) cudaGraphSetConditional(a.cond, 0);
}

__global__ void sssp_round_end_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    if (a.hdr->done) return;
    if (round_end(a.hdr) && a.use_cond) cudaGraphSetConditional(a.cond, 0);
}

__global__ void sssp_init_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.V; v += stride) init_vertex(a, v);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.queue[0][0] = a.source;
        a.hdr->frontier_edges = a.row_off[a.source + 1] - a.row_off[a.source];  // round 0's frontier
    }
}

// ---- partitioned (out-of-HBM) solves -------------------------------------

// Per-partition HyTM metrics of this round's frontier: active vertices,
// active edges (out-edges of active vertices), zero-copy requests
// ceil(deg * 4 / 128) and alignment overhead (row start not 128-byte aligned
// in the logical id array), as in the reference's cost model
// (src/transfer/hytm_cost_model.cpp:330-452).  Shared-memory histograms,
// one global atomic per CTA and partition.
constexpr uint32_t kMaxParts = 1024;

__global__ void __launch_bounds__(kSSThreads) sssp_part_stats_kernel(const SSArgs *__restrict__ args, uint32_t parts,
                                                                     PartMetrics *out) {
    __shared__ unsigned long long s_m[4 * kMaxParts];
    const SSArgs a = *args;
    for (uint32_t i = threadIdx.x; i < 4 * parts; i += blockDim.x) s_m[i] = 0;
    __syncthreads();
    const RoundView rv = round_view(a);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rv.qn; i += gridDim.x * blockDim.x) {
        const uint32_t v = rv.q[i];
        const uint32_t p = v >> a.part_shift;
        const uint64_t off = a.row_off[v];
        const uint64_t deg = a.row_off[v + 1] - off;
        atomicAdd(&s_m[4 * p + 0], 1ull);
        if (deg) {
            atomicAdd(&s_m[4 * p + 1], static_cast<unsigned long long>(deg));
            atomicAdd(&s_m[4 * p + 2], static_cast<unsigned long long>((deg * 4 + 127) / 128));
            if ((off * 4) % 128) atomicAdd(&s_m[4 * p + 3], 1ull);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 4 * parts; i += blockDim.x)
        if (s_m[i]) atomicAdd(reinterpret_cast<unsigned long long *>(out) + i, s_m[i]);
}

// Frontier vertices whose partition is compacted this round.
__global__ void sssp_compacted_list_kernel(const SSArgs *__restrict__ args, uint32_t *list, uint32_t *count) {
    const SSArgs a = *args;
    const RoundView rv = round_view(a);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rv.qn; i += gridDim.x * blockDim.x) {
        const uint32_t v = rv.q[i];
        if (a.loc[v >> a.part_shift].mode == kLocCompacted) append(list, count, v);
    }
}

// Expands the packed rows of compacted partitions (row i: vertex verts[i],
// edges [index[i], index[i+1]) of the packed cols / weights).
template <int WK>
__global__ void __launch_bounds__(kSSThreads) sssp_expand_packed_kernel(const SSArgs *__restrict__ args,
                                                                        CompactPayload pk) {
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done) return;
    const RoundView rv = round_view(a);
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * kSSThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kSSThreads) >> 5;
    unsigned long long relaxed = 0, improved = 0;
    for (uint64_t w = gwarp; w * 32 < pk.rows; w += nwarps) {
        const uint64_t i = w * 32 + lane;
        uint32_t deg = 0, d = a.inf;
        uint64_t off = 0;
        if (i < pk.rows) {
            off = pk.index[i];
            deg = static_cast<uint32_t>(pk.index[i + 1] - off);
            d = __ldcg(a.dist + pk.verts[i]);
            relaxed += deg;
        }
        uint32_t incl = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t base = 0; base < total; base += 32 * kEdgeBatch) {
            uint32_t u[kEdgeBatch], nd[kEdgeBatch], du[kEdgeBatch];
#pragma unroll
            for (int k = 0; k < kEdgeBatch; ++k) {
                const uint32_t j = base + 32 * k + lane;
                uint32_t lo = 0;
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1) {
                    const uint32_t probe = __shfl_sync(0xffffffffu, incl, lo + step - 1);
                    if (probe <= j) lo += step;
                }
                const uint32_t o_incl = __shfl_sync(0xffffffffu, incl, lo);
                const uint32_t o_deg = __shfl_sync(0xffffffffu, deg, lo);
                const uint64_t o_off = __shfl_sync(0xffffffffu, off, lo);
                const uint32_t o_d = __shfl_sync(0xffffffffu, d, lo);
                u[k] = 0;
                nd[k] = a.inf;
                if (j < total) {
                    const uint64_t e = o_off + (j - (o_incl - o_deg));
                    u[k] = dev::ld_stream(pk.cols + e);
                    nd[k] = extend<WK>(o_d, edge_weight<WK>(pk.weights, e));
                }
            }
#pragma unroll
            for (int k = 0; k < kEdgeBatch; ++k) du[k] = __ldcg(a.dist + u[k]);
            relax_batch<kEdgeBatch>(a, rv, u, nd, du, lane, improved);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) relaxed += __shfl_xor_sync(0xffffffffu, relaxed, o);
    if (lane == 0 && relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
}

// Row skipping in pull sweeps (env HYT_SSSP_PULL_SKIP, 0 = off; default on).
bool sssp_pull_skip() {
    static bool on = [] {
        const char *e = std::getenv("HYT_SSSP_PULL_SKIP");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Smallest of n weights (bit patterns of u32 or non-negative f32 weights;
// -0.0 counts as 0) into *out, which starts at all ones.
__global__ void min_weight_kernel(const uint32_t *__restrict__ w, uint64_t n, uint32_t f32, uint32_t *out) {
    uint32_t m = 0xFFFFFFFFu;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t x = __ldcs(w + i);
        m = min(m, f32 ? (x & 0x7FFFFFFFu) : x);
    }
    m = __reduce_min_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) atomicMin(out, m);
}

// The graph's smallest CSC weight, found once per graph.
uint32_t graph_min_in_weight(GraphImpl &g, bool f32, cudaStream_t s) {
    if (!g.min_in_weight_ready) {
        Scratch<uint32_t> m(1, s);
        HYT_CUDA(cudaMemsetAsync(m.get(), 0xFF, sizeof(uint32_t), s));
        min_weight_kernel<<<grid_for(g.E, 256, 148 * 8), 256, 0, s>>>(g.in_weights.get(), g.E, f32 ? 1u : 0u,
                                                                       m.get());
        HYT_CUDA(cudaGetLastError());
        uint32_t local = 0;
        uint32_t *h = g.host_scratch.ptr ? reinterpret_cast<uint32_t *>(g.host_scratch.ptr) : &local;
        HYT_CUDA(cudaMemcpyAsync(h, m.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        g.min_in_weight = *h;
        g.min_in_weight_ready = true;
    }
    return g.min_in_weight;
}

// Pull sweeps when the frontier's out-edges exceed E / div (env
// HYT_SSSP_PULL_DIV, 0 = never; default 4: a sweep reads every in-edge once,
// which costs about what pushing a quarter of them does).
uint32_t sssp_pull_div() {
    static uint32_t div = [] {
        const char *e = std::getenv("HYT_SSSP_PULL_DIV");
        return e ? static_cast<uint32_t>(std::strtoul(e, nullptr, 10)) : 4u;
    }();
    return div;
}

template <int WK>
int pull_grid(bool staged, unsigned smem) {
    static bool attr = false;
    if (!attr) {
        HYT_CUDA(cudaFuncSetAttribute(sssp_pull_kernel<WK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaFuncSetAttribute(sssp_pull_staged_kernel<WK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        attr = true;
    }
    int per_sm = 0;
    if (staged)
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_pull_staged_kernel<WK>,
                                                               stage::kStageThreads, smem));
    else
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_pull_kernel<WK>, kPullThreads, smem));
    return sm_count() * std::max(per_sm, 1);
}

// Staged pull sweeps when asked for (HYT_STAGED=1) and the graph's tiles
// fit a staging slot.
bool pull_use_staged(const GraphImpl &g) {
    return stage::staged_requested() && g.tile_cost <= kStageTileMax && g.pull_tasks.get() &&
           stage::staged_shared_bytes(g.num_hot) <= kPRSmemMax;
}

template <int WK>
int expand_grid() {
    static int g = 0;
    if (g == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_expand_kernel<WK>, kSSThreads, 0));
        g = sm_count() * std::max(per_sm, 1);
    }
    return g;
}

template <int WK>
void sssp_solve(GraphImpl &g, uint32_t source, uint32_t delta, uint32_t max_rounds, uint32_t flags, cudaStream_t s,
                uint32_t *dist_out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    if (g.dist.count < V) g.dist.allocate(V);
    if (g.stamp.count < 2 * V) g.stamp.allocate(2 * V);
    for (int i = 0; i < 2; ++i) {
        if (g.queue[i].count < V) g.queue[i].allocate(V);
        if (g.far[i].count < V) g.far[i].allocate(V);
    }
    // each frontier vertex appears once per round: <= V rows, E/kHubChunk + V chunks
    const uint64_t hub_cap = V + g.E / kHubChunk + 2;
    if (g.hub_tasks.count < hub_cap) g.hub_tasks.allocate(hub_cap);
    const size_t sb = 512 + sizeof(SSHeader);
    if (g.sssp_state.count < sb) g.sssp_state.allocate(sb);
    SSArgs *d_args = reinterpret_cast<SSArgs *>(g.sssp_state.get());
    SSHeader *hdr = reinterpret_cast<SSHeader *>(g.sssp_state.get() + 256);

    SSArgs a{};
    a.row_off = g.row_offsets.get();
    a.cols = g.cols.get();
    a.weights = g.weights.get();
    a.dist = g.dist.get();
    a.stamp = g.stamp.get();
    a.fstamp = g.stamp.get() + V;
    for (int i = 0; i < 2; ++i) {
        a.queue[i] = g.queue[i].get();
        a.far[i] = g.far[i].get();
    }
    a.hubs = g.hub_tasks.get();
    a.hdr = hdr;
    a.V = static_cast<uint32_t>(V);
    a.source = source;
    a.inf = (WK == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
    a.num_edges = g.E;
    // pull sweeps need the CSC (and its weights) and a single bucket
    const bool pull_ok = (g.flags & HYT_GRAPH_PULL) && (WK == HYT_WEIGHTS_NONE || g.in_weights.get()) &&
                         delta == kNoDelta && g.E > 0;
    a.pull_div = pull_ok ? sssp_pull_div() : 0u;
    PullGraph pg{};
    if (a.pull_div) {
        pg.in_off = g.in_offsets.get();
        pg.in_src = g.in_sources.get();
        pg.in_w = g.in_weights.get();
        pg.tile_start = g.tile_start.get();
        pg.long_rows = g.long_rows.get();
        pg.chunk_tasks = g.chunk_tasks.get();
        pg.hot_vertex = g.hot_vertex.get();
        pg.tasks = g.pull_tasks.get();
        pg.num_tiles = g.num_tiles;
        pg.num_chunks = g.num_chunks;
        pg.tile_cost = g.tile_cost;
        pg.num_hot = g.num_hot;
    }
    const bool staged = a.pull_div && pull_use_staged(g);
    // row skipping (register-path sweeps): the smallest edge weight bounds
    // what any in-edge adds
    if (a.pull_div && !staged && sssp_pull_skip()) {
        a.skip_rows = 1;
        a.min_w = (WK == HYT_WEIGHTS_NONE) ? 1u : graph_min_in_weight(g, WK == HYT_WEIGHTS_F32, s);
    }
    const unsigned pull_smem =
        staged ? static_cast<unsigned>(stage::staged_shared_bytes(g.num_hot))
               : static_cast<unsigned>((g.num_hot + kPullThreads / 32 * (2 * size_t(g.tile_cost) + 8)) * 4);
    const int pgrid = a.pull_div ? pull_grid<WK>(staged, pull_smem) : 0;
    const void *pull_fn = staged ? reinterpret_cast<const void *>(sssp_pull_staged_kernel<WK>)
                                 : reinterpret_cast<const void *>(sssp_pull_kernel<WK>);

    SSHeader h0{};
    h0.qsize[0] = 1;
    h0.max_rounds = max_rounds;
    h0.delta = delta;
    h0.threshold = (WK == HYT_WEIGHTS_F32 || delta == kNoDelta) ? 0xFFFFFFFFu : delta;
    const bool far_pile = h0.threshold != 0xFFFFFFFFu;  // labels above the threshold wait in the far pile

    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    const int grid = expand_grid<WK>();
    // The round loop's shape; an instantiated loop of the same shape (kept
    // with the graph object) is launched again instead of being rebuilt.
    struct LoopKey {
        int wk, grid, pgrid;
        uint32_t far_pile, pull_div, staged, pull_smem;
        const void *args;
        PullGraph pg;
    } key;
    std::memset(&key, 0, sizeof(key));
    key.wk = WK;
    key.grid = grid;
    key.pgrid = pgrid;
    key.far_pile = far_pile;
    key.pull_div = a.pull_div;
    key.staged = staged;
    key.pull_smem = pull_smem;
    key.args = d_args;
    key.pg = pg;
    LoopGraph &loop = g.sssp_loop;
    const bool reuse = use_graph && loop.matches(&key, sizeof(key));
    if (use_graph && !reuse) {
        loop.reset();
        HYT_CUDA(cudaGraphCreate(&loop.graph, 0));
        HYT_CUDA(cudaGraphConditionalHandleCreate(&loop.cond, loop.graph, 1, cudaGraphCondAssignDefault));
    }
    if (use_graph) {
        a.cond = loop.cond;
        a.use_cond = 1;
    }

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaMemcpyAsync(hdr, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    sssp_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 1, hot = 0;
    double kernel_ms = 0.0;
    // split (finite bucket width), expand, hub, pull sweep + round close or round end
    const uint32_t per_round = (far_pile ? 1u : 0u) + 3u + (a.pull_div ? 1u : 0u);

    if (use_graph) {
        if (!reuse) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = loop.cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cnode;
            HYT_CUDA(cudaGraphAddNode(&cnode, loop.graph, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            void *kargs[] = {&d_args};
            cudaKernelNodeParams kp = {};
            kp.kernelParams = kargs;
            kp.blockDim = dim3(kSSThreads);
            kp.gridDim = dim3(grid);
            cudaGraphNode_t prev = nullptr, node;
            auto add = [&](const void *f, dim3 gd, dim3 bd, unsigned smem, void **params) {
                kp.func = const_cast<void *>(f);
                kp.gridDim = gd;
                kp.blockDim = bd;
                kp.sharedMemBytes = smem;
                kp.kernelParams = params;
                HYT_CUDA(cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
                prev = node;
            };
            void *pargs[] = {&d_args, &pg};
            // one bucket (no threshold): the far pile stays empty, nothing to split
            if (far_pile) add(reinterpret_cast<void *>(sssp_split_kernel), dim3(grid), dim3(kSSThreads), 0, kargs);
            add(reinterpret_cast<void *>(sssp_expand_kernel<WK>), dim3(grid), dim3(kSSThreads), 0, kargs);
            add(reinterpret_cast<void *>(sssp_hub_kernel<WK>), dim3(grid), dim3(kSSThreads), 0, kargs);
            if (a.pull_div) {
                add(pull_fn, dim3(pgrid), dim3(staged ? stage::kStageThreads : kPullThreads), pull_smem, pargs);
                add(reinterpret_cast<void *>(sssp_round_close_kernel), dim3(grid), dim3(kSSThreads), 0, kargs);
            } else {
                add(reinterpret_cast<void *>(sssp_round_end_kernel), dim3(1), dim3(1), 0, kargs);
            }
            HYT_CUDA(cudaGraphInstantiate(&loop.exec, loop.graph, 0));
            loop.set_key(&key, sizeof(key));
        }
        HYT_CUDA(cudaGraphLaunch(loop.exec, s));
    } else {
        EventTimer kt;
        for (uint32_t r = 0; r < max_rounds; ++r) {
            if (flags & HYT_RUN_PROFILE) kt.start(s);
            if (far_pile) sssp_split_kernel<<<grid, kSSThreads, 0, s>>>(d_args);
            sssp_expand_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
            sssp_hub_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
            if (a.pull_div) {
                if (staged)
                    sssp_pull_staged_kernel<WK><<<pgrid, stage::kStageThreads, pull_smem, s>>>(d_args, pg);
                else
                    sssp_pull_kernel<WK><<<pgrid, kPullThreads, pull_smem, s>>>(d_args, pg);
            }
            if (a.pull_div)
                sssp_round_close_kernel<<<grid, kSSThreads, 0, s>>>(d_args);  // frontier-edge count + round end
            if (flags & HYT_RUN_PROFILE) kt.stop(s);
            if (!a.pull_div) sssp_round_end_kernel<<<1, 1, 0, s>>>(d_args);
            HYT_CUDA(cudaGetLastError());
            launches += per_round;
            hot += a.pull_div ? per_round : per_round - 1;
            uint32_t done = 0;
            HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            if (flags & HYT_RUN_PROFILE) kernel_ms += kt.ms();
            if (done) break;
        }
    }
    SSHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (use_graph) launches += per_round * h.round;
    if (h.error) fail(HYT_E_TIMEOUT, "SSSP: a bounded wait for a staged copy ran out");
    if (dist_out) graph_emit(g, dist_out, g.dist.get(), s);
    if (stats) {
        stats->iterations = h.round;
        stats->converged = h.converged;
        stats->residual = 0.0;
        stats->device_ms = total_ms;
        stats->kernel_ms = kernel_ms;
        stats->kernel_launches = hot;
        stats->total_launches = launches;
        stats->edges_processed = h.relaxations;
        stats->vertices_processed = h.frontier_total;
        // per frontier vertex: 8 B offset pair (read twice) + 4 B label +
        // 4 B queue entry; per edge: 4 B column + 4 B weight + 4 B label.
        stats->algorithmic_bytes = 16ull * h.frontier_total + 12ull * h.relaxations;
    }
}

}  // namespace

uint32_t sssp_default_delta(const GraphImpl &g) {
    // Measured on R-MAT scale 24 (bucket widths 4 .. infinity): with batched
    // relaxations the extra rounds of narrow buckets cost more than the
    // relaxations they save, so the default is one bucket (frontier
    // Bellman-Ford).  Callers pick a finite width with params.delta; a
    // graph's 2x-mean-weight width is kept in g.default_delta for that.
    (void)g;
    return kNoDelta;
}

void sssp_run(GraphImpl &g, const hyt_sssp_params &p, uint32_t *dist_out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PUSH");
    if (p.source >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    // Termination is guaranteed (labels only decrease, weights >= 0); the
    // round cap is a safety bound on the device loop.
    const uint64_t cap = std::min<uint64_t>(4 * g.V + 1024, 0x7FFFFFFFull);
    const uint32_t max_rounds = p.max_rounds ? p.max_rounds : static_cast<uint32_t>(cap);
    const uint32_t delta = p.delta ? p.delta : sssp_default_delta(g);
    const uint32_t src = graph_vertex(g, p.source, s);
    switch (g.weight_kind) {
        case HYT_WEIGHTS_NONE: sssp_solve<HYT_WEIGHTS_NONE>(g, src, delta, max_rounds, p.flags, s, dist_out, stats); break;
        case HYT_WEIGHTS_U32: sssp_solve<HYT_WEIGHTS_U32>(g, src, delta, max_rounds, p.flags, s, dist_out, stats); break;
        case HYT_WEIGHTS_F32: sssp_solve<HYT_WEIGHTS_F32>(g, src, kNoDelta, max_rounds, p.flags, s, dist_out, stats); break;
        default: fail(HYT_E_INTERNAL, "unknown weight kind");
    }
}

// Round loop of an out-of-HBM solve: per round the frontier's partition
// metrics go to the source, which places every partition's edges (resident,
// staged, mapped host memory) or compacts them; then the usual expansion.
template <int WK>
static void sssp_partitioned_solve(GraphImpl &g, PushSource &src, uint32_t source, uint32_t max_rounds,
                                   cudaStream_t s, uint32_t *dist_out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    const size_t P = src.parts();
    if (P == 0 || P > kMaxParts) fail(HYT_E_UNSUPPORTED, "partitioned SSSP supports 1..1024 partitions");
    if (g.dist.count < V) g.dist.allocate(V);
    if (g.stamp.count < 2 * V) g.stamp.allocate(2 * V);
    for (int i = 0; i < 2; ++i) {
        if (g.queue[i].count < V) g.queue[i].allocate(V);
        if (g.far[i].count < V) g.far[i].allocate(V);
    }
    const uint64_t hub_cap = V + g.E / kHubChunk + 2;
    if (g.hub_tasks.count < hub_cap) g.hub_tasks.allocate(hub_cap);
    const size_t sb = 512 + sizeof(SSHeader);
    if (g.sssp_state.count < sb) g.sssp_state.allocate(sb);
    SSArgs *d_args = reinterpret_cast<SSArgs *>(g.sssp_state.get());
    SSHeader *hdr = reinterpret_cast<SSHeader *>(g.sssp_state.get() + 256);
    DeviceArray<EdgeLoc> d_loc(P);
    DeviceArray<PartMetrics> d_metrics(P);
    DeviceArray<uint32_t> d_list(V + 1);
    uint32_t *d_count = d_list.get() + V;
    PinnedArray<uint32_t> h_list;

    SSArgs a{};
    a.row_off = g.row_offsets.get();
    a.dist = g.dist.get();
    a.stamp = g.stamp.get();
    a.fstamp = g.stamp.get() + V;
    for (int i = 0; i < 2; ++i) {
        a.queue[i] = g.queue[i].get();
        a.far[i] = g.far[i].get();
    }
    a.hubs = g.hub_tasks.get();
    a.hdr = hdr;
    a.V = static_cast<uint32_t>(V);
    a.source = source;
    a.inf = (WK == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
    a.loc = d_loc.get();
    a.part_shift = src.part_shift();
    SSHeader h0{};
    h0.qsize[0] = 1;
    h0.max_rounds = max_rounds;
    h0.delta = kNoDelta;
    h0.threshold = 0xFFFFFFFFu;

    const int grid = expand_grid<WK>();
    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaMemcpyAsync(hdr, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    sssp_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 1;
    std::vector<PartMetrics> metrics(P);
    RoundPlan plan;
    for (uint32_t r = 0; r < max_rounds; ++r) {
        sssp_split_kernel<<<grid, kSSThreads, 0, s>>>(d_args);
        HYT_CUDA(cudaMemsetAsync(d_metrics.get(), 0, P * sizeof(PartMetrics), s));
        sssp_part_stats_kernel<<<sm_count() * 2, kSSThreads, 0, s>>>(d_args, static_cast<uint32_t>(P), d_metrics.get());
        HYT_CUDA(cudaGetLastError());
        HYT_CUDA(cudaMemcpyAsync(metrics.data(), d_metrics.get(), P * sizeof(PartMetrics), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        src.plan_round(metrics, plan);
        launches += 2;
        for (size_t w = 0; w < plan.waves.size(); ++w) {
            src.enter_wave(w, s);
            HYT_CUDA(cudaMemcpyAsync(d_loc.get(), plan.waves[w].data(), P * sizeof(EdgeLoc), cudaMemcpyHostToDevice,
                                     s));
            sssp_expand_kernel<WK, true><<<grid, kSSThreads, 0, s>>>(d_args);
            sssp_hub_kernel<WK, true><<<grid, kSSThreads, 0, s>>>(d_args);
            HYT_CUDA(cudaGetLastError());
            HYT_CUDA(cudaMemsetAsync(&hdr->hub_count, 0, sizeof(uint32_t), s));
            src.leave_wave(w, s);
            launches += 2;
        }
        if (plan.compacted) {
            HYT_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint32_t), s));
            sssp_compacted_list_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args, d_list.get(), d_count);
            HYT_CUDA(cudaGetLastError());
            uint32_t n = 0;
            HYT_CUDA(cudaMemcpyAsync(&n, d_count, sizeof(n), cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            if (n) {
                if (h_list.count < n) h_list.allocate(std::max<size_t>(n, 1u << 20));
                HYT_CUDA(cudaMemcpyAsync(h_list.ptr, d_list.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                HYT_CUDA(cudaStreamSynchronize(s));
                const CompactPayload pk = src.compact(h_list.ptr, n, s);
                sssp_expand_packed_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args, pk);
                HYT_CUDA(cudaGetLastError());
                launches += 2;
            }
        }
        sssp_round_end_kernel<<<1, 1, 0, s>>>(d_args);
        HYT_CUDA(cudaGetLastError());
        ++launches;
        src.end_round(s);
        uint32_t done = 0;
        HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (done) break;
    }
    SSHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (dist_out) copy_from_device(dist_out, g.dist.get(), V * sizeof(uint32_t), s);
    if (stats) {
        stats->iterations = h.round;
        stats->converged = h.converged;
        stats->device_ms = total_ms;
        stats->total_launches = launches;
        stats->edges_processed = h.relaxations;
        stats->vertices_processed = h.frontier_total;
        stats->algorithmic_bytes = 16ull * h.frontier_total + 12ull * h.relaxations;
    }
}

void sssp_partitioned(GraphImpl &g, PushSource &src, uint32_t source, uint32_t max_rounds, cudaStream_t s,
                      uint32_t *dist_out, hyt_run_stats *stats) {
    if (source >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
    const uint64_t cap = std::min<uint64_t>(4 * g.V + 1024, 0x7FFFFFFFull);
    const uint32_t rounds = max_rounds ? max_rounds : static_cast<uint32_t>(cap);
    switch (g.weight_kind) {
        case HYT_WEIGHTS_NONE: sssp_partitioned_solve<HYT_WEIGHTS_NONE>(g, src, source, rounds, s, dist_out, stats); break;
        case HYT_WEIGHTS_U32: sssp_partitioned_solve<HYT_WEIGHTS_U32>(g, src, source, rounds, s, dist_out, stats); break;
        case HYT_WEIGHTS_F32: sssp_partitioned_solve<HYT_WEIGHTS_F32>(g, src, source, rounds, s, dist_out, stats); break;
        default: fail(HYT_E_INTERNAL, "unknown weight kind");
    }
}

}  // namespace hyt

namespace hyt {

// ===========================================================================
// SSSP that allocates nothing: hyt_sssp_noalloc (include/hyt/capi.h).
//
// For callers that cannot call cudaMalloc: a host application whose caching
// allocator already holds the device's free memory, a latency-critical loop
// that must not pay cudaMalloc's implicit device synchronisation, or a plugin
// host that forbids its components to allocate.  The caller passes its CSR
// and the output label array in device memory; every other buffer the solver
// needs lives in one file-scope __device__ array of kNoAllocScratchBytes that
// each GPU loading this library holds until the process exits.
//
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current and caches it; make that
// first call before any stream capture.  Every call shares the array and it
// keeps the previous call's contents; whatever must start at zero is cleared
// by the call itself.  Calls whose work overlaps on the GPU (other streams,
// other threads) race on the array.
// ===========================================================================
namespace {

constexpr uint64_t kNoAllocMaxVertices = HYT_NOALLOC_MAX_VERTICES;
constexpr uint64_t kNoAllocMaxEdges = HYT_NOALLOC_MAX_EDGES;
constexpr uint64_t kNoAllocHubCap = kNoAllocMaxVertices + kNoAllocMaxEdges / kHubChunk + 2;
// args (256 B) | header (256 B) | check word (64 B) | stamp+fstamp u32[2V] |
// queue u32[2][V] | far u32[2][V] | hub tasks uint2[hub cap]
constexpr size_t kNoAllocHeadBytes = 1024;
// head: arguments at 0, header at 256, validation flags at 512
static_assert(sizeof(SSArgs) <= 256 && sizeof(SSHeader) <= 256, "no-alloc head layout");
constexpr size_t kNoAllocScratchBytes =
    kNoAllocHeadBytes + 6 * sizeof(uint32_t) * kNoAllocMaxVertices + sizeof(uint2) * kNoAllocHubCap;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_address[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code
// the name g_noalloc_scratch is only a host-side stand-in, never passed to a
// kernel.
unsigned char *noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) fail(HYT_E_UNSUPPORTED, "hyt_sssp_noalloc: device ordinal too large");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_address[device]) {
        void *p = nullptr;
        HYT_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_address[device] = p;
    }
    return static_cast<unsigned char *>(g_noalloc_address[device]);
}

// Rejects malformed CSR input before any kernel indexes with it.
__global__ void noalloc_check_kernel(const uint64_t *off, const uint32_t *cols, const uint32_t *w, uint32_t wkind,
                                     uint64_t V, uint64_t E, uint32_t *bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t i0 = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t b = 0;
    for (uint64_t v = i0; v < V; v += stride)
        if (off[v + 1] < off[v]) b |= 1u;
    for (uint64_t e = i0; e < E; e += stride) {
        if (cols[e] >= V) b |= 2u;
        if (wkind == HYT_WEIGHTS_F32) {
            const float x = __uint_as_float(w[e]);
            if (!(x >= 0.0f) || isinf(x)) b |= 4u;
        }
    }
    if (i0 == 0 && (off[0] != 0 || off[V] != E)) b |= 1u;
    if (b) atomicOr(bad, b);
}

template <int WK>
void sssp_noalloc_solve(const hyt_csr &csr, uint32_t source, uint32_t *dist, cudaStream_t s, unsigned char *scratch,
                        hyt_run_stats *stats) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    SSArgs *d_args = reinterpret_cast<SSArgs *>(scratch);
    SSHeader *hdr = reinterpret_cast<SSHeader *>(scratch + 256);
    uint32_t *check = reinterpret_cast<uint32_t *>(scratch + 512);
    uint32_t *stamp = reinterpret_cast<uint32_t *>(scratch + kNoAllocHeadBytes);
    uint32_t *queue0 = stamp + 2 * kNoAllocMaxVertices;
    uint32_t *queue1 = queue0 + kNoAllocMaxVertices;
    uint32_t *far0 = queue1 + kNoAllocMaxVertices;
    uint32_t *far1 = far0 + kNoAllocMaxVertices;
    uint2 *hubs = reinterpret_cast<uint2 *>(far1 + kNoAllocMaxVertices);

    HYT_CUDA(cudaMemsetAsync(check, 0, sizeof(uint32_t), s));
    noalloc_check_kernel<<<grid_for(std::max(V, E), 256, 148 * 8), 256, 0, s>>>(
        csr.row_offsets, csr.column_indices, static_cast<const uint32_t *>(csr.weights), WK, V, E, check);
    HYT_CUDA(cudaGetLastError());
    uint32_t bad = 0;
    HYT_CUDA(cudaMemcpyAsync(&bad, check, sizeof(bad), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (bad & 1u) fail(HYT_E_INVALID, "hyt_sssp_noalloc: row offsets must start at 0, be non-decreasing and end at E");
    if (bad & 2u) fail(HYT_E_INVALID, "hyt_sssp_noalloc: column index contains an invalid destination vertex ID");
    if (bad & 4u) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");

    SSArgs a{};
    a.row_off = csr.row_offsets;
    a.cols = csr.column_indices;
    a.weights = static_cast<const uint32_t *>(csr.weights);
    a.dist = dist;
    a.stamp = stamp;
    a.fstamp = stamp + kNoAllocMaxVertices;
    a.queue[0] = queue0;
    a.queue[1] = queue1;
    a.far[0] = far0;
    a.far[1] = far1;
    a.hubs = hubs;
    a.hdr = hdr;
    a.V = static_cast<uint32_t>(V);
    a.source = source;
    a.inf = (WK == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;
    a.use_cond = 0;

    SSHeader h0{};  // every counter of the round state starts at zero
    h0.qsize[0] = 1;
    h0.delta = kNoDelta;
    h0.threshold = 0xFFFFFFFFu;
    const uint32_t max_rounds = static_cast<uint32_t>(4 * V + 1024);
    h0.max_rounds = max_rounds;

    const int grid = expand_grid<WK>();
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaMemcpyAsync(hdr, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    sssp_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 2;
    for (uint32_t r = 0; r < max_rounds; ++r) {
        sssp_split_kernel<<<grid, kSSThreads, 0, s>>>(d_args);
        sssp_expand_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
        sssp_hub_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
        sssp_round_end_kernel<<<1, 1, 0, s>>>(d_args);
        HYT_CUDA(cudaGetLastError());
        launches += 4;
        uint32_t done = 0;
        HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (done) break;
    }
    SSHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = h.round;
        stats->converged = h.converged;
        stats->total_launches = launches;
        stats->edges_processed = h.relaxations;
        stats->vertices_processed = h.frontier_total;
        stats->algorithmic_bytes = 16ull * h.frontier_total + 12ull * h.relaxations;
    }
}

}  // namespace

void sssp_noalloc(const hyt_csr &csr, uint32_t source, uint32_t *dist_out, void *stream, hyt_run_stats *stats) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (V == 0) fail(HYT_E_INVALID, "SSSP requires at least one vertex");
    if (V > kNoAllocMaxVertices || E > kNoAllocMaxEdges)
        fail(HYT_E_INVALID, "hyt_sssp_noalloc: graph exceeds the fixed scratch capacity (at most " +
                                std::to_string(kNoAllocMaxVertices) + " vertices and " +
                                std::to_string(kNoAllocMaxEdges) + " edges); use hyt_sssp for larger graphs");
    if (source >= V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    if (csr.weight_kind > HYT_WEIGHTS_F32) fail(HYT_E_INVALID, "unknown weight_kind");
    int device = 0;
    HYT_CUDA(cudaGetDevice(&device));
    // Every array is dereferenced by kernels on the current device: host
    // memory and another GPU's memory are refused before any launch
    // (column_indices and weights are read only when there are edges).
    const bool edges = E > 0, weights = edges && csr.weight_kind != HYT_WEIGHTS_NONE;
    const std::pair<const void *, const char *> arrays[] = {{csr.row_offsets, "row_offsets"},
                                                           {csr.column_indices, edges ? "column_indices" : nullptr},
                                                           {csr.weights, weights ? "weights" : nullptr},
                                                           {dist_out, "dist_out"}};
    for (const auto &[ptr, name] : arrays) {
        if (!name) continue;
        int owner = -1;
        const PointerPlace place = pointer_place(ptr, device, &owner);
        if (place == PointerPlace::kHost)
            fail(HYT_E_INVALID, std::string("hyt_sssp_noalloc: ") + name +
                                    " must be device memory of the current device (got host memory)");
        if (place == PointerPlace::kOtherDevice)
            fail(HYT_E_INVALID, std::string("hyt_sssp_noalloc: ") + name + " is device memory of GPU " +
                                    std::to_string(owner) + ", not of the current device " +
                                    std::to_string(device));
    }
    unsigned char *scratch = noalloc_scratch(device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (csr.weight_kind) {
        case HYT_WEIGHTS_NONE: sssp_noalloc_solve<HYT_WEIGHTS_NONE>(csr, source, dist_out, s, scratch, stats); break;
        case HYT_WEIGHTS_U32: sssp_noalloc_solve<HYT_WEIGHTS_U32>(csr, source, dist_out, s, scratch, stats); break;
        default: sssp_noalloc_solve<HYT_WEIGHTS_F32>(csr, source, dist_out, s, scratch, stats); break;
    }
}

}  // namespace hyt
