// Device building blocks of pull PageRank / personalized PageRank, shared
// by the single-query solver (pagerank.cu), the partitioned out-of-HBM
// solver and the batched multi-query engine (batch.cu): the per-row
// finalisation, the batched contribution gather, and the two task kinds
// (merge-path tile of short rows; chunk of a long row merged by its last
// arriving warp).  Semantics are described at the top of pagerank.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "graph.cuh"

namespace hyt {
namespace prc {

#ifndef HYT_PR_WARP_ROW
#define HYT_PR_WARP_ROW 64
#endif
constexpr uint32_t kWarpRowDegree = HYT_PR_WARP_ROW;  // rows with more in-edges are summed by a whole warp

struct PRHeader {
    uint32_t iter;       // iterations completed
    uint32_t done;
    uint32_t converged;
    uint32_t error;      // 1: a bounded wait for a staged copy ran out
    double last_residual;
};

// Fixed-order reduction of an iteration's residual and dangling mass.
// Every task owns a slot: tile k -> num_long + k, long row i -> i (written
// by the warp that finalizes the row) -- a plain store, nothing waits on it.
// After the iteration's tasks, pr_reduce_kernel sums each group of
// kSlotGroup slots in slot order (a fixed block tree), and its last block
// sums the group sums in group order and closes the iteration.  The result
// is the same for any grid, launch split or arrival order.  The counter
// only grows (each iteration adds the reduce grid), so it is cleared once
// per solve.
constexpr uint32_t kSlotGroup = 1024;

struct PRSlots {
    double2 *slot;          // [num_slots] (residual, dangling)
    double2 *group_sum;     // [num_groups]
    uint32_t *blocks_done;  // [1] reduce blocks finished, over the whole solve
    uint32_t num_slots, num_groups;
};

// Device-resident arguments (a cached CUDA graph reads them every launch).
struct PRArgs {
    const uint64_t *in_off;
    const uint32_t *in_src;
    const uint32_t *out_deg;
    const uint32_t *tile_start;
    const LongRow *long_rows;
    const uint2 *chunk_tasks;
    const uint32_t *hot_vertex;  // [num_hot] vertices cached in shared memory
    uint32_t num_hot;
    uint32_t tile_cost;
    float *rank[2];
    float *contrib[2];
    float2 *partial;
    uint32_t *ticket;
    PRHeader *hdr;
    double *residual;        // [max_iter]
    double *dangling;        // [max_iter + 1]
    uint64_t num_tiles;
    uint32_t num_chunks;
    uint32_t V;
    float damping;
    float base;         // PR: (1-d)/n
    float tolerance;
    uint32_t max_iter;
    uint32_t source;    // PPR
    uint32_t personalized;
    cudaGraphConditionalHandle cond;
    uint32_t use_cond;
    PRSlots red;        // fixed-order residual / dangling reduction (single-query solver)
    const uint4 *tasks; // pull task descriptors (staged solver)
};

struct PRState {
    // per-iteration scalars
    float damping, base, teleport_scale;
    float dshare;  // PR: d * dangling / n
    float tele;    // PPR: (1-d) + d * dangling
    uint32_t source;
    bool personalized;
};

// Row r's next rank, contribution, L1 change and dangling share from its
// in-edge sum, given its current rank `old` and out-degree `od`.
__device__ __forceinline__ void finalize_row_with(const PRState &ps, uint32_t r, float sum, float old, uint32_t od,
                                                  float *nxt, float *cnxt, double &res, double &dang) {
    float nx;
    if (ps.personalized) {
        nx = __fmul_rn(ps.damping, sum);
        if (r == ps.source) nx = __fadd_rn(ps.tele, nx);
    } else {
        nx = __fadd_rn(ps.dshare, __fmul_rn(ps.damping, sum));
    }
    res += fabs(static_cast<double>(nx) - static_cast<double>(old));
    nxt[r] = nx;
    cnxt[r] = od ? __fdiv_rn(nx, static_cast<float>(od)) : 0.0f;
    if (od == 0) dang += static_cast<double>(nx);
}

__device__ __forceinline__ void finalize_row(const PRArgs &a, const PRState &ps, uint32_t r, float sum,
                                             const float *cur, float *nxt, float *cnxt, double &res, double &dang) {
    float nx;
    if (ps.personalized) {
        nx = __fmul_rn(ps.damping, sum);
        if (r == ps.source) nx = __fadd_rn(ps.tele, nx);
    } else {
        nx = __fadd_rn(ps.dshare, __fmul_rn(ps.damping, sum));
    }
    const float old = cur[r];
    res += fabs(static_cast<double>(nx) - static_cast<double>(old));
    nxt[r] = nx;
    const uint32_t od = a.out_deg[r];
    cnxt[r] = od ? __fdiv_rn(nx, static_cast<float>(od)) : 0.0f;
    if (od == 0) dang += static_cast<double>(nx);
}

// Gathers the contributions of edges [lo, hi) of the in-source array.
// Lane l of the warp takes edges lo + base + 32k + l (k < kBatch): each of
// the kBatch id loads is one coalesced 128-byte access, and because the
// sources of an in-row are sorted, the 32 addresses of each gather
// instruction are ascending and neighbouring lanes often share an L2 sector
// (dense for hub-heavy rows).  All kBatch gathers of a lane are issued
// before any is consumed.  Edges past hi yield 0 and read a clamped address.
#ifndef HYT_PR_BATCH
#define HYT_PR_BATCH 16
#endif
constexpr int kBatch = HYT_PR_BATCH;

// kSmemHot: hot sources (tagged ids) read their contribution from the
// CTA's shared-memory copy s_hot; otherwise from ccur[hot_vertex[slot]].
// One pass of kK = 4 * kG batches (edges src[base + 32k + lane], k < kK).
template <int kK, bool kSmemHot, class Sink>
__device__ __forceinline__ void gather_pass(const uint32_t *src, uint32_t base, uint32_t n, const float *ccur,
                                            const float *s_hot, const uint32_t *hot_vertex, uint64_t pol, int lane,
                                            Sink &sink) {
    uint32_t id[kK];
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const uint32_t i = base + 32 * k + lane;
        id[k] = (i < n) ? dev::ld_stream(src + i) : 0u;
    }
    float v[kK];
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        v[k] = 0.0f;
        if (!(id[k] & kHotTag)) v[k] = dev::ld_keep(ccur + id[k], pol);
    }
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        if (id[k] & kHotTag) {
            if constexpr (kSmemHot) {
                v[k] = s_hot[id[k] & ~kHotTag];
            } else {
                v[k] = ccur[hot_vertex[id[k] & ~kHotTag]];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const uint32_t i = base + 32 * k + lane;
        if (i < n) sink(i, v[k]);
    }
}

// A pass over the last, partial batch group issues only the 4-batch groups
// that hold edges (a warp-uniform choice), so short tiles do not pay for
// kBatch gather slots; the edges and their order are the same.
template <bool kSmemHot, class Sink>
__device__ __forceinline__ void gather_span(const uint32_t *in_src, const float *ccur, const float *s_hot,
                                            const uint32_t *hot_vertex, uint64_t lo, uint64_t hi, uint64_t pol,
                                            int lane, Sink &&sink) {
    static_assert(kBatch % 4 == 0 && kBatch >= 4, "batches come in groups of 4");
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    const uint32_t *src = in_src + lo;
    for (uint32_t base = 0; base < n; base += 32 * kBatch) {
        const uint32_t groups = (n - base + 127) / 128;  // 4-batch groups holding edges
        if (groups >= kBatch / 4)
            gather_pass<kBatch, kSmemHot>(src, base, n, ccur, s_hot, hot_vertex, pol, lane, sink);
        else if (groups == 1)
            gather_pass<4, kSmemHot>(src, base, n, ccur, s_hot, hot_vertex, pol, lane, sink);
        else if (groups == 2)
            gather_pass<8, kSmemHot>(src, base, n, ccur, s_hot, hot_vertex, pol, lane, sink);
        else
            gather_pass<(kBatch >= 12 ? 12 : kBatch), kSmemHot>(src, base, n, ccur, s_hot, hot_vertex, pol, lane,
                                                                sink);
    }
}

// Stop rule of iteration `it` (thread 0 of the last CTA, or the separate
// end kernel): residual <= tolerance or the iteration cap.
__device__ __forceinline__ void end_iteration(const PRArgs &a, uint32_t it) {
    const double r = atomicAdd(&a.residual[it], 0.0);
    const uint32_t n_it = it + 1;
    const bool conv = r <= static_cast<double>(a.tolerance);
    a.hdr->last_residual = r;
    a.hdr->iter = n_it;
    if (conv || n_it >= a.max_iter) {
        a.hdr->done = 1;
        a.hdr->converged = conv ? 1u : 0u;
        if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
    }
}


// Ends iteration `it` on the device (any thread): the stop rule with the
// iteration's reduced residual.
__device__ __forceinline__ void close_iteration(const PRArgs &a, uint32_t it, double residual, double dangling) {
    a.residual[it] = residual;
    a.dangling[it + 1] = dangling;
    const uint32_t n_it = it + 1;
    const bool conv = residual <= static_cast<double>(a.tolerance);
    a.hdr->last_residual = residual;
    a.hdr->iter = n_it;
    if (conv || n_it >= a.max_iter) {
        a.hdr->done = 1;
        a.hdr->converged = conv ? 1u : 0u;
        if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
    }
}

// Records task slot `slot`'s (res, dang); lane 0 stores, no wait.
__device__ __forceinline__ void slot_store(const PRArgs &a, uint32_t slot, double res, double dang, int lane) {
    if (lane == 0) a.red.slot[slot] = make_double2(res, dang);
}

// Solver scalars of an iteration whose dangling mass (sum of x over
// out-degree-0 vertices) is dmass.
__device__ __forceinline__ PRState make_state(const PRArgs &a, double dmass) {
    PRState ps;
    ps.damping = a.damping;
    ps.source = a.source;
    ps.personalized = a.personalized != 0;
    ps.dshare = __fadd_rn(a.base, static_cast<float>(static_cast<double>(a.damping) * dmass / static_cast<double>(a.V)));
    ps.tele = static_cast<float>((1.0 - static_cast<double>(a.damping)) + static_cast<double>(a.damping) * dmass);
    return ps;
}

// Rank buffers of iteration `it` (Jacobi double buffering by parity).
struct PRBuffers {
    const float *cur, *ccur;
    float *nxt, *cnxt;
};

__device__ __forceinline__ PRBuffers buffers(const PRArgs &a, uint32_t it) {
    PRBuffers b;
    b.cur = (it & 1) ? a.rank[1] : a.rank[0];
    b.nxt = (it & 1) ? a.rank[0] : a.rank[1];
    b.ccur = (it & 1) ? a.contrib[1] : a.contrib[0];
    b.cnxt = (it & 1) ? a.contrib[0] : a.contrib[1];
    return b;
}

// Chunk task `ci` (index into a.chunk_tasks): a kLongChunk-edge slice of a
// long row.  The warp stores its compensated partial; the last arriving
// warp of the row merges every partial in chunk order (lane j takes chunks
// j, j+32, ...) and finalizes the row.  Returns the row's long-row index
// when this warp finalized it (lane 0 holds res/dang), else ~0u.  Must be
// called by all 32 lanes.
template <bool kSmemHot>
__device__ __forceinline__ uint32_t chunk_task(const PRArgs &a, const PRState &ps, const PRBuffers &b,
                                               const uint32_t *in_src, const float *s_hot, uint64_t ci, uint64_t pol,
                                               int lane, double &res, double &dang,
                                               const uint4 *prefetch = nullptr) {
    const uint2 t = a.chunk_tasks[ci];
    const LongRow L = a.long_rows[t.x];
    const uint64_t rb = a.in_off[L.row], re = a.in_off[L.row + 1];
    const uint64_t lo = rb + uint64_t(t.y) * kLongChunk;
    const uint64_t hi = (lo + kLongChunk < re) ? lo + kLongChunk : re;
    dev::CSum acc;
    gather_span<kSmemHot>(in_src, b.ccur, s_hot, a.hot_vertex, lo, hi, pol, lane,
                          [&](uint32_t, float v) { acc.add(v); });
    if (prefetch) prefetch_task(*prefetch, in_src, nullptr, lane);
    acc = dev::warp_reduce(acc);
    uint32_t last = 0;
    if (lane == 0) {
        a.partial[L.first_chunk + t.y] = make_float2(acc.s, acc.c);
        __threadfence();
        const uint32_t tk = atomicAdd(&a.ticket[t.x], 1u) + 1u;
        last = (tk % L.num_chunks == 0) ? 1u : 0u;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return ~0u;
    __threadfence();
    dev::CSum row;
    for (uint32_t j = lane; j < L.num_chunks; j += 32) {
        const float2 p = __ldcg(a.partial + L.first_chunk + j);
        dev::CSum x;
        x.s = p.x;
        x.c = p.y;
        row.merge(x);
    }
    row = dev::warp_reduce(row);
    if (lane == 0) finalize_row(a, ps, L.row, row.value(), b.cur, b.nxt, b.cnxt, res, dang);
    return t.x;
}

// Tile task k: rows [tile_start[k], tile_start[k+1]) minus a long last row
// (chunked).  The tile's contributions are gathered into the warp's
// shared-memory slice sv, then summed lane-per-row (in-degree <
// kWarpRowDegree) or warp-per-row, in edge order.  Must be called by all 32
// lanes.
// prefetch (optional): the warp's next pull task, whose edge lines are
// warmed in L2 once this task's gathers are issued.
template <bool kSmemHot>
__device__ __forceinline__ void tile_task(const PRArgs &a, const PRState &ps, const PRBuffers &b,
                                          const uint32_t *in_src, const float *s_hot, float *sv, uint64_t k,
                                          uint64_t pol, int lane, double &res, double &dang,
                                          const uint4 *prefetch = nullptr) {
    const uint32_t r0 = a.tile_start[k];
    const uint32_t r1 = a.tile_start[k + 1];
    if (r0 == r1) return;
    const uint64_t last_b = a.in_off[r1 - 1], last_e = a.in_off[r1];
    const uint32_t rl = (last_e - last_b >= a.tile_cost) ? r1 - 1 : r1;  // long last row is chunked
    const uint64_t e0 = a.in_off[r0];
    const uint64_t e1 = (rl == r1) ? last_e : last_b;
    // the first 32 rows' bounds (relative to e0), ranks and out-degrees,
    // loaded before the gathers so that they arrive with them
    uint32_t lo_p = 0, hi_p = 0, od_p = 0;
    float old_p = 0.0f;
    if (r0 + lane < rl) {
        lo_p = static_cast<uint32_t>(a.in_off[r0 + lane] - e0);
        hi_p = static_cast<uint32_t>(a.in_off[r0 + lane + 1] - e0);
        old_p = b.cur[r0 + lane];
        od_p = a.out_deg[r0 + lane];
    }
    gather_span<kSmemHot>(in_src, b.ccur, s_hot, a.hot_vertex, e0, e1, pol, lane,
                          [&](uint32_t i, float v) { sv[i] = v; });
    if (prefetch) prefetch_task(*prefetch, in_src, nullptr, lane);
    __syncwarp();
    for (uint32_t rb = r0; rb < rl; rb += 32) {
        const uint32_t r = rb + lane;
        const bool active = r < rl;
        uint32_t lo = lo_p, hi = hi_p, od = od_p;
        float old = old_p;
        if (rb != r0) {
            lo = active ? static_cast<uint32_t>(a.in_off[r] - e0) : 0u;
            hi = active ? static_cast<uint32_t>(a.in_off[r + 1] - e0) : 0u;
            old = active ? b.cur[r] : 0.0f;
            od = active ? a.out_deg[r] : 0u;
        }
        if (active && hi - lo < kWarpRowDegree) {
            dev::CSum acc;
            for (uint32_t x = lo; x < hi; ++x) acc.add(sv[x]);
            finalize_row_with(ps, r, acc.value(), old, od, b.nxt, b.cnxt, res, dang);
        }
        uint32_t big = __ballot_sync(0xffffffffu, active && (hi - lo >= kWarpRowDegree));
        while (big) {
            const int src = __ffs(big) - 1;
            big &= big - 1;
            const uint32_t bb = __shfl_sync(0xffffffffu, lo, src);
            const uint32_t ee = __shfl_sync(0xffffffffu, hi, src);
            const float o_src = __shfl_sync(0xffffffffu, old, src);
            const uint32_t d_src = __shfl_sync(0xffffffffu, od, src);
            dev::CSum acc;
            for (uint32_t x = bb + lane; x < ee; x += 32) acc.add(sv[x]);
            acc = dev::warp_reduce(acc);
            if (lane == 0) finalize_row_with(ps, rb + src, acc.value(), o_src, d_src, b.nxt, b.cnxt, res, dang);
        }
    }
    __syncwarp();
}

}  // namespace prc
}  // namespace hyt
