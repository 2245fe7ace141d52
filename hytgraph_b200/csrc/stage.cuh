// Per-warp staging pipeline of the pull kernels (PageRank iterations and
// SSSP pull sweeps over an in-HBM CSC).  A warp walks its pull tasks
// (graph.cuh descriptors) as units -- a tile, or a kUnitEdges-edge piece of
// a long-row chunk -- and stages each unit's source ids into shared memory
// with one bulk copy (cp.async.bulk, completion on an mbarrier), one unit
// ahead of the unit it is working on.  Ids then cost no registers and no
// load latency on the warp's critical path; the warp's registers go to the
// dependent gathers instead.
//
// Sources are this GPU's own memory only (no multicast).
//
// The staged kernels are opt-in (HYT_STAGED=1, which also selects
// kStageTileMax-unit tiles so that a tile fits one slot).  On R-MAT graphs
// the register-path kernels with 512-unit tiles ran faster: the pull
// kernels are bound by instruction issue over the dependent gathers, not by
// the id stream, and half-size tiles leave half of each unit's gather
// slots and row lanes idle.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>

#include <cstdint>

#include "bulk.cuh"
#include "graph.cuh"

namespace hyt::stage {

constexpr uint32_t kUnitEdges = 512;  // edges of one staged unit (a tile, or a piece of a chunk)
constexpr uint32_t kSlotWords = 520;  // unit + 16-byte alignment at both ends, in 4-byte words
#ifndef HYT_STAGE_SLOTS
#define HYT_STAGE_SLOTS 3
#endif
#ifndef HYT_STAGE_WARPS
#define HYT_STAGE_WARPS 24
#endif
constexpr int kStageSlots = HYT_STAGE_SLOTS;  // staging slots per warp: units staged ahead + 1
constexpr int kStageWarps = HYT_STAGE_WARPS;  // warps per CTA of the staged kernels
constexpr int kStageThreads = kStageWarps * 32;
static_assert(kStageSlots >= 2, "at least double buffering");
// A tile's edges: the rows starting inside a tile span < tile_cost merge
// units, and its last short row adds < tile_cost more, so < 2 * tile_cost.
static_assert(2 * kStageTileMax - 1 + 6 <= kSlotWords, "a tile's edges must fit one staging slot");
static_assert(kLongChunk % kUnitEdges == 0, "chunks split into whole units");

// The unit a slot holds (written by lane 0 when its copy is issued).
struct UnitMeta {
    uint4 d;     // task descriptor
    uint64_t t;  // task index
    uint32_t j;  // unit of the task
    uint32_t pad;
};

// Dynamic shared memory of the staged kernels: per-warp mbarriers, unit
// records and slots, then the hot-source table.
constexpr size_t kStageBars = size_t(kStageWarps) * kStageSlots * sizeof(uint64_t);
constexpr size_t kStageMeta = size_t(kStageWarps) * kStageSlots * sizeof(UnitMeta);
constexpr size_t kStageHead = ((kStageBars + kStageMeta + 127) / 128) * 128;
constexpr size_t kStageBytes = kStageHead + size_t(kStageWarps) * kStageSlots * kSlotWords * 4;

inline size_t staged_shared_bytes(uint32_t num_hot) { return kStageBytes + size_t(num_hot) * 4; }

// HYT_STAGED=1: in-HBM PageRank and SSSP pull sweeps use the staged kernels.
inline bool staged_requested() {
    static const bool on = [] {
        const char *e = std::getenv("HYT_STAGED");
        return e && e[0] == '1';
    }();
    return on;
}

#ifdef __CUDACC__

// This warp's barriers, unit records and slots in the kernel's dynamic
// shared memory (kStageBytes from its start); lane 0 initialises the
// barriers.
struct WarpStage {
    uint64_t *bars;
    UnitMeta *meta;
    uint32_t *slots;
};
__device__ __forceinline__ WarpStage warp_stage(unsigned char *smem, int warp, int lane) {
    WarpStage w;
    w.bars = reinterpret_cast<uint64_t *>(smem) + warp * kStageSlots;
    w.meta = reinterpret_cast<UnitMeta *>(smem + kStageBars) + warp * kStageSlots;
    w.slots = reinterpret_cast<uint32_t *>(smem + kStageHead) + size_t(warp) * kStageSlots * kSlotWords;
    if (lane == 0)
        for (int i = 0; i < kStageSlots; ++i) bulk::mbar_init(w.bars + i);
    bulk::fence_barrier_init();
    __syncwarp();
    return w;
}

// Edge range [lo, hi) of unit j of task d.
struct Unit {
    uint64_t lo, hi;
};
__device__ __forceinline__ Unit unit_of(uint4 d, uint32_t j) {
    const uint64_t e0 = task_first_edge(d), n = task_edges(d);
    const uint64_t lo = e0 + uint64_t(j) * kUnitEdges;
    return Unit{lo, (lo + kUnitEdges < e0 + n) ? lo + kUnitEdges : e0 + n};
}
__device__ __forceinline__ uint32_t units_of(uint4 d) {
    return task_is_chunk(d) ? (task_edges(d) + kUnitEdges - 1) / kUnitEdges : 1u;
}

// Lane 0 announces and issues the bulk copy of unit u's ids (16-byte
// aligned: the span rounded out to whole 4-id groups, which the 16 bytes of
// tail padding behind every id array keep in bounds) into `slot`.
__device__ __forceinline__ void stage_unit(const uint32_t *in_src, Unit u, uint32_t *slot, uint64_t *bar, uint64_t pol,
                                           int lane) {
    if (lane == 0) {
        const uint64_t a0 = u.lo & ~uint64_t(3), a1 = (u.hi + 3) & ~uint64_t(3);
        const uint32_t bytes = static_cast<uint32_t>(a1 - a0) * 4u;
        bulk::mbar_arrive_expect_tx(bar, bytes);
        if (bytes) bulk::copy_g2s(slot, in_src + a0, bytes, bar, pol);
    }
}

// Drives one warp through its tasks (first, first + stride, ... < total):
// keeps kStageSlots - 1 units staged ahead of the one being worked on, and
// calls consume(d, task, j, units, slot words, first staged edge) for each
// unit once its ids have landed.  false: a wait ran out (the copies still in
// flight have been waited for, within the same budget).
template <class Consume>
__device__ __forceinline__ bool stage_pipeline(const uint4 *tasks, const uint32_t *in_src, uint64_t first,
                                               uint64_t stride, uint64_t total, const WarpStage &ws, int lane,
                                               Consume &&consume) {
    if (first >= total) return true;
    const uint64_t pol = bulk::policy_evict_first();
    // producer cursor: the next unit to stage
    uint4 pd = tasks[first];
    uint64_t pt = first, nt = first + stride;
    uint4 dn = nt < total ? tasks[nt] : make_uint4(0, 0, 0, 0);
    uint32_t pj = 0;
    bool pvalid = true;
    auto produce = [&](int slot) {
        if (lane == 0) ws.meta[slot] = UnitMeta{pd, pt, pj, 0};
        stage_unit(in_src, unit_of(pd, pj), ws.slots + slot * kSlotWords, ws.bars + slot, pol, lane);
        if (pj + 1 < units_of(pd)) {
            ++pj;
        } else {
            pvalid = nt < total;
            pd = dn;
            pt = nt;
            pj = 0;
            if (pvalid) {
                nt += stride;
                dn = nt < total ? tasks[nt] : make_uint4(0, 0, 0, 0);
            }
        }
    };
    uint64_t issued = 0, consumed = 0;
    for (int s = 0; s < kStageSlots && pvalid; ++s, ++issued) produce(s);
    __syncwarp();
    uint32_t phase = 0;
    while (consumed < issued) {
        const int s = static_cast<int>(consumed % kStageSlots);
        if (!bulk::mbar_wait(ws.bars + s, (phase >> s) & 1u)) {
            for (uint64_t c = consumed + 1; c < issued; ++c) {  // copies still in flight
                const int o = static_cast<int>(c % kStageSlots);
                bulk::mbar_wait(ws.bars + o, (phase >> o) & 1u);
            }
            return false;
        }
        phase ^= 1u << s;
        const UnitMeta m = ws.meta[s];
        const Unit u = unit_of(m.d, m.j);
        consume(m.d, m.t, m.j, units_of(m.d), ws.slots + s * kSlotWords, u.lo & ~uint64_t(3));
        bulk::fence_proxy_async_smem();  // this slot's generic accesses before its next bulk copy
        __syncwarp();
        ++consumed;
        if (pvalid) {
            produce(s);
            ++issued;
            __syncwarp();
        }
    }
    return true;
}

// The same walk without staging, for graphs whose tiles exceed a slot:
// consume(d, task, j, units, in_src, 0) for every unit of every task, the
// consumer reading ids from global memory in place.
template <class Consume>
__device__ __forceinline__ void direct_tasks(const uint4 *tasks, const uint32_t *in_src, uint64_t first,
                                             uint64_t stride, uint64_t total, Consume &&consume) {
    for (uint64_t t = first; t < total; t += stride) {
        const uint4 d = tasks[t];
        const uint32_t nu = units_of(d);
        for (uint32_t j = 0; j < nu; ++j) consume(d, t, j, nu, in_src, uint64_t(0));
    }
}

#endif  // __CUDACC__

}  // namespace hyt::stage
