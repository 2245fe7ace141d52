// Device building blocks of frontier SSSP, shared by the single-query
// solver (sssp.cu), the partitioned out-of-HBM solver and the batched
// multi-query engine (batch.cu): round state, label relaxation with
// warp-aggregated frontier appends, warp-centric row expansion and the
// round-end rule.  Semantics are described at the top of sssp.cu.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "hybrid.cuh"
#include "hyt/capi.h"

namespace hyt {
namespace ssc {

namespace cg = cooperative_groups;

constexpr int kSSThreads = 256;
constexpr uint32_t kHubDegree = 64;   // rows at least this long become warp tasks
constexpr uint32_t kHubChunk = 512;   // edges per warp task
constexpr uint32_t kNoDelta = 0xFFFFFFFFu;
#ifndef HYT_SS_EXPAND_BATCH
#define HYT_SS_EXPAND_BATCH 8
#endif
#ifndef HYT_SS_HUB_BATCH
#define HYT_SS_HUB_BATCH 8
#endif
constexpr int kEdgeBatch = HYT_SS_EXPAND_BATCH;  // 32-edge batches in flight per warp (short rows)
constexpr int kHubBatch = HYT_SS_HUB_BATCH;      // the same for hub tasks

struct SSHeader {
    uint32_t round;      // rounds completed
    uint32_t done;
    uint32_t converged;
    uint32_t phase;      // far-pile generation
    uint32_t pending;    // 1: this round starts by splitting the far pile
    uint32_t threshold;  // near/far boundary T
    uint32_t old_threshold;
    uint32_t delta;
    uint32_t qsize[2];   // near frontier sizes, by round parity
    uint32_t fsize[2];   // far pile sizes, by phase parity
    uint32_t hub_count;
    uint32_t max_rounds;
    unsigned long long relaxations;     // edges relaxed
    unsigned long long frontier_total;  // frontier vertices expanded
    unsigned long long frontier_edges;  // out-edges of this round's frontier (pull-capable solves)
    uint32_t pull_rounds;               // rounds run as pull sweeps
    uint32_t error;                     // 1: a bounded wait for a staged copy ran out
    unsigned long long frontier_edges_next;  // out-edges of the next frontier, summed at round close
    uint32_t close_ticket;                   // blocks of the round-close kernel finished
    uint32_t fmin;      // lowest label in this round's frontier (pull-capable solves with row skipping)
    uint32_t fmin_inv;  // ~(lowest label) of the next frontier, gathered at round close
    uint32_t pad;
};

struct SSArgs {
    const uint64_t *row_off;
    const uint32_t *cols;
    const uint32_t *weights;
    uint32_t *dist;
    uint32_t *stamp;   // round in whose frontier a vertex sits
    uint32_t *fstamp;  // far-pile generation that holds a vertex
    uint32_t *queue[2];
    uint32_t *far[2];
    uint2 *hubs;
    SSHeader *hdr;
    uint32_t V;
    uint32_t source;
    uint32_t inf;
    uint32_t use_cond;
    cudaGraphConditionalHandle cond;
    const EdgeLoc *loc;   // per-partition edge location (partitioned solves)
    uint32_t part_shift;  // partition of vertex v = v >> part_shift
    uint32_t pull_div;    // > 0: a round whose frontier has more than E / pull_div out-edges is a pull sweep
    uint64_t num_edges;
    uint32_t skip_rows;   // 1: pull sweeps skip rows whose label no in-edge can lower (needs fmin)
    uint32_t min_w;       // smallest edge weight (bit pattern; 1 when unweighted)
};

// True when this round runs as a pull sweep over the CSC instead of a push
// expansion (decided from the frontier's out-edge count, identically by
// every kernel of the round).
__device__ __forceinline__ bool pull_round(const SSArgs &a) {
    if (!a.pull_div) return false;
    const unsigned long long fe = *(volatile const unsigned long long *)&a.hdr->frontier_edges;
    return fe * a.pull_div > a.num_edges;
}

template <int WK>
__device__ __forceinline__ uint32_t edge_weight(const uint32_t *w, uint64_t e) {
    if constexpr (WK == HYT_WEIGHTS_NONE) {
        return 1u;
    } else {
        return dev::ld_stream(w + e);
    }
}

template <int WK>
__device__ __forceinline__ uint32_t extend(uint32_t d, uint32_t w) {
    if constexpr (WK == HYT_WEIGHTS_F32) {
        return __float_as_uint(__fadd_rn(__uint_as_float(d), __uint_as_float(w)));
    } else {
        const uint64_t s = uint64_t(d) + w;
        return s >= 0xFFFFFFFFull ? 0xFFFFFFFEu : static_cast<uint32_t>(s);
    }
}

__device__ __forceinline__ void append(uint32_t *list, uint32_t *size, uint32_t v) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(size, g.size());
    base = g.shfl(base, 0);
    list[base + g.thread_rank()] = v;
}

// Per-round view of the header, read once by every thread.
struct RoundView {
    uint32_t r, qn, threshold, next_stamp, far_stamp;
    const uint32_t *q;
    uint32_t *qnext, *qnext_size, *far, *far_size;
};

__device__ __forceinline__ RoundView round_view(const SSArgs &a) {
    const SSHeader *h = a.hdr;
    RoundView rv;
    rv.r = *(volatile const uint32_t *)&h->round;
    const uint32_t odd = rv.r & 1;
    rv.qn = *(volatile const uint32_t *)(odd ? &h->qsize[1] : &h->qsize[0]);
    rv.q = odd ? a.queue[1] : a.queue[0];
    rv.qnext = odd ? a.queue[0] : a.queue[1];
    rv.qnext_size = odd ? &a.hdr->qsize[0] : &a.hdr->qsize[1];
    rv.threshold = *(volatile const uint32_t *)&h->threshold;
    rv.next_stamp = rv.r + 1;
    // During a split round the far pile of the next phase is already active.
    const uint32_t p = *(volatile const uint32_t *)&h->phase + *(volatile const uint32_t *)&h->pending;
    rv.far = (p & 1) ? a.far[1] : a.far[0];
    rv.far_size = (p & 1) ? &a.hdr->fsize[1] : &a.hdr->fsize[0];
    rv.far_stamp = p + 1;
    return rv;
}

// Appends each lane's entries vals[k] with bit k set in `mask` to a list,
// with one atomic per warp.  Must be called by all 32 lanes.
template <int K>
__device__ __forceinline__ void warp_append(uint32_t *list, uint32_t *size, const uint32_t (&vals)[K], uint32_t mask,
                                            int lane) {
    const uint32_t cnt = __popc(mask);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    uint32_t base = 0;
    if (lane == 31) base = atomicAdd(size, total);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - cnt;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((mask >> k) & 1u) list[base + __popc(mask & ((1u << k) - 1u))] = vals[k];
}

// Relaxes K candidate edges per lane with all atomics of a phase in flight
// together: atomicMin on every improving label, then the stamp exchange of
// every success, then one warp-aggregated append per list.  nd[k] >= du[k]
// (including padding lanes, whose nd is the infinity label) is a no-op.
// Must be called by all 32 lanes.
template <int K>
__device__ __forceinline__ void relax_batch(const SSArgs &a, const RoundView &rv, const uint32_t (&u)[K],
                                            const uint32_t (&nd)[K], const uint32_t (&du)[K], int lane,
                                            unsigned long long &improved) {
    uint32_t old[K];
#pragma unroll
    for (int k = 0; k < K; ++k) old[k] = (nd[k] < du[k]) ? atomicMin(a.dist + u[k], nd[k]) : 0u;
    uint32_t st[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        st[k] = 0;
        if (nd[k] < old[k])
            st[k] = (nd[k] < rv.threshold) ? atomicExch(a.stamp + u[k], rv.next_stamp)
                                           : atomicExch(a.fstamp + u[k], rv.far_stamp);
    }
    uint32_t nmask = 0, fmask = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (nd[k] < old[k]) {
            ++improved;
            if (nd[k] < rv.threshold) {
                if (st[k] != rv.next_stamp) nmask |= 1u << k;
            } else if (st[k] != rv.far_stamp) {
                fmask |= 1u << k;
            }
        }
    }
    warp_append<K>(rv.qnext, rv.qnext_size, u, nmask, lane);
    warp_append<K>(rv.far, rv.far_size, u, fmask, lane);
}


// Expands frontier positions [i0, i0 + 32) of rv (lane l takes i0 + l):
// rows shorter than hub_degree are walked by the warp as one combined edge
// list, 32 edges at a time with kEdgeBatch batches in flight; longer rows
// are handed to hub(v, chunks) as kHubChunk-edge tasks.  HYB: the edges of
// a vertex's partition are reached through a.loc (out-of-HBM solves).
// Must be called by all 32 lanes.
// kB: 32-edge batches in flight.  The in-HBM solver's expansion takes 16;
// the batch engine's and the out-of-HBM expansion keep kEdgeBatch (with 16
// their kernels spill registers).
template <int WK, bool HYB, int kB = kEdgeBatch, class HubSink>
__device__ __forceinline__ void expand_warp(const SSArgs &a, const RoundView &rv, uint32_t i0, int lane,
                                            uint32_t hub_degree, unsigned long long &relaxed,
                                            unsigned long long &improved, HubSink &&hub) {
    const uint32_t i = i0 + lane;
    uint32_t deg = 0, d = a.inf;
    uint64_t off = 0;
    const uint32_t *vc = a.cols, *vw = a.weights;  // edge arrays of this lane's vertex
    if (i < rv.qn) {
        const uint32_t v = rv.q[i];
        off = a.row_off[v];
        uint64_t full = a.row_off[v + 1] - off;
        if constexpr (HYB) {
            const EdgeLoc L = a.loc[v >> a.part_shift];
            vc = L.cols;
            vw = L.weights;
            if (L.mode != kLocDirect || v < L.vlo || v >= L.vhi) full = 0;
        }
        d = __ldcg(a.dist + v);
        relaxed += full;
        if (full >= hub_degree) {
            hub(v, static_cast<uint32_t>((full + kHubChunk - 1) / kHubChunk));
        } else {
            deg = static_cast<uint32_t>(full);
        }
    }
    // inclusive prefix of the 32 short degrees
    uint32_t incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t base = 0; base < total; base += 32 * kB) {
        uint32_t u[kB], nd[kB], du[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            const uint32_t j = base + 32 * k + lane;
            // owner = first lane whose inclusive prefix exceeds j
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
            const uint32_t *oc = a.cols, *ow = a.weights;
            if constexpr (HYB) {
                oc = reinterpret_cast<const uint32_t *>(
                    __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(vc), lo));
                ow = reinterpret_cast<const uint32_t *>(
                    __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(vw), lo));
            }
            u[k] = 0;
            nd[k] = a.inf;
            if (j < total) {
                const uint64_t e = o_off + (j - (o_incl - o_deg));
                u[k] = dev::ld_stream(oc + e);
                nd[k] = extend<WK>(o_d, edge_weight<WK>(ow, e));
            }
        }
#pragma unroll
        for (int k = 0; k < kB; ++k) du[k] = __ldcg(a.dist + u[k]);
        relax_batch<kB>(a, rv, u, nd, du, lane, improved);
    }
}

// One kHubChunk-edge slice (chunk c) of frontier row v, edges read from
// hc / hw (global-edge-indexed).  Must be called by all 32 lanes.
template <int WK>
__device__ __forceinline__ void hub_chunk(const SSArgs &a, const RoundView &rv, const uint32_t *hc,
                                          const uint32_t *hw, uint32_t v, uint32_t c, int lane,
                                          unsigned long long &improved) {
    const uint64_t rb = a.row_off[v], re = a.row_off[v + 1];
    const uint64_t b = rb + uint64_t(c) * kHubChunk;
    const uint32_t len = static_cast<uint32_t>(((b + kHubChunk < re) ? b + kHubChunk : re) - b);
    const uint32_t d = __ldcg(a.dist + v);
    for (uint32_t base = 0; base < len; base += 32 * kHubBatch) {
        uint32_t u[kHubBatch], nd[kHubBatch], du[kHubBatch];
#pragma unroll
        for (int k = 0; k < kHubBatch; ++k) {
            const uint32_t j = base + 32 * k + lane;
            u[k] = 0;
            nd[k] = a.inf;
            if (j < len) {
                u[k] = dev::ld_stream(hc + b + j);
                nd[k] = extend<WK>(d, edge_weight<WK>(hw, b + j));
            }
        }
#pragma unroll
        for (int k = 0; k < kHubBatch; ++k) du[k] = __ldcg(a.dist + u[k]);
        relax_batch<kHubBatch>(a, rv, u, nd, du, lane, improved);
    }
}

// Far-pile entry i of a pending split: settled entries are dropped, those
// below the new threshold join this round's near frontier, the rest move to
// the next far pile.
__device__ __forceinline__ void split_entry(const SSArgs &a, uint32_t i) {
    const SSHeader *h = a.hdr;
    const uint32_t r = h->round, p = h->phase;
    const uint32_t lo = h->old_threshold, hi = h->threshold;
    const uint32_t *src = (p & 1) ? a.far[1] : a.far[0];
    uint32_t *dst = (p & 1) ? a.far[0] : a.far[1];
    uint32_t *dst_size = (p & 1) ? &a.hdr->fsize[0] : &a.hdr->fsize[1];
    uint32_t *near = (r & 1) ? a.queue[1] : a.queue[0];
    uint32_t *near_size = (r & 1) ? &a.hdr->qsize[1] : &a.hdr->qsize[0];
    const uint32_t v = src[i];
    const uint32_t d = __ldcg(a.dist + v);
    if (d < lo) return;  // settled in an earlier phase
    if (d < hi) {
        a.stamp[v] = r;
        append(near, near_size, v);
    } else {
        a.fstamp[v] = p + 2;
        append(dst, dst_size, v);
    }
}

// Closes a round (single thread): swaps the frontiers, starts a far-pile
// split when the near frontier ran dry, and applies the stop rule.
// Returns true when the solve is finished.
__device__ __forceinline__ bool round_end(SSHeader *h) {
    const uint32_t r = h->round;
    const uint32_t n_next = h->qsize[(r + 1) & 1];
    h->frontier_total += h->qsize[r & 1];
    h->qsize[r & 1] = 0;
    h->hub_count = 0;
    h->frontier_edges = 0;
    h->round = r + 1;
    if (h->pending) {  // the split of this round consumed the old far pile
        h->fsize[h->phase & 1] = 0;
        h->phase += 1;
        h->pending = 0;
    }
    bool finish = false, conv = false;
    if (n_next == 0) {
        if (h->fsize[h->phase & 1] == 0) {
            finish = conv = true;
        } else {
            h->pending = 1;
            h->old_threshold = h->threshold;
            const uint64_t t = uint64_t(h->threshold) + h->delta;
            h->threshold = t >= 0xFFFFFFFFull ? 0xFFFFFFFFu : static_cast<uint32_t>(t);
        }
    }
    if (!finish && r + 1 >= h->max_rounds) finish = true;
    if (finish) {
        h->done = 1;
        h->converged = conv ? 1u : 0u;
    }
    return finish;
}

// Initial labels of one vertex.
__device__ __forceinline__ void init_vertex(const SSArgs &a, uint32_t v) {
    const bool s = (v == a.source);
    a.dist[v] = s ? 0u : a.inf;
    a.stamp[v] = s ? 0u : 0xFFFFFFFFu;
    a.fstamp[v] = 0xFFFFFFFFu;
}

}  // namespace ssc
}  // namespace hyt
