// Packed personalized PageRank: up to 8 queries on one graph share every
// pass over the CSC (hyt_ppr_multi).
//
// Each query keeps the single-source definition (hyt_ppr; the oracle's
// personalized PageRank):
//   x' = d * sum_{u->v} x_u / deg(u) + [v == s] * ((1 - d) + d * dangling),
//   d = 1 - restart, x_0 = e_s, stop after the step whose L1 change is
//   <= tolerance.
// The 8 lanes of a vertex are stored together (32 bytes), so one in-edge
// costs one source id and one 32-byte sector of contributions for all 8
// queries, instead of 8 id reads and 8 scattered gathers.  A thread takes
// four of a vertex's queries with one 16-byte load per in-edge: short rows
// 16 per warp (two threads per row), longer rows by the whole warp in 16
// edge slots; sums are FP64, folded with shuffles in a fixed order, and
// rows at or above the graph's long-row threshold use its 4096-edge chunk
// tasks, summed per row in chunk order.  The thread layout does not depend
// on how many lanes are in use,
// so a query's result is the same bit for bit alone or packed with others.
// A lane whose step met its tolerance stops (its values are carried
// unchanged) while the others continue.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "graph.cuh"
#include "prims.cuh"
#include "scratch.cuh"
#include "solvers.cuh"
#include "stage.cuh"

namespace hyt {
namespace {

constexpr int kLanes = 8;
constexpr int kPartBlocks = 512;

// c[u][l] = x[u][l] / deg(u) (0 when dangling); per-block partial sums of
// the dangling values, per lane.
__global__ void ppr8_prep_kernel(const uint32_t *__restrict__ deg, const float *__restrict__ x, uint64_t V,
                                 float *__restrict__ c, double *__restrict__ dpart) {
    __shared__ double s_part[kLanes][8];
    double acc[kLanes] = {};
    for (uint64_t u = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; u < V; u += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t d = deg[u];
        const float4 a = reinterpret_cast<const float4 *>(x)[2 * u];
        const float4 b = reinterpret_cast<const float4 *>(x)[2 * u + 1];
        const float v[kLanes] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        float o[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            o[l] = d ? __fdiv_rn(v[l], float(d)) : 0.0f;
            if (!d) acc[l] += v[l];
        }
        reinterpret_cast<float4 *>(c)[2 * u] = make_float4(o[0], o[1], o[2], o[3]);
        reinterpret_cast<float4 *>(c)[2 * u + 1] = make_float4(o[4], o[5], o[6], o[7]);
    }
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int l = 0; l < kLanes; ++l) {
        double a = acc[l];
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) a += __shfl_xor_sync(0xffffffffu, a, sh);
        if ((threadIdx.x & 31) == 0) s_part[l][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double a = 0.0;
        for (int w = 0; w < 8; ++w) a += s_part[threadIdx.x][w];
        dpart[blockIdx.x * kLanes + threadIdx.x] = a;
    }
}

// Sums over in-edges [b, e) of c[u][4h .. 4h + 3], h = t % 2: thread t
// takes edge slot t / 2 (16 slots) and adds its edges b + t/2, b + t/2 + 16,
// ... in that order, four queries at a time from one 16-byte load
// (kQuadInFlight edges loaded before any is added); the slots are then folded by
// shuffles, so every thread of half h holds the four sums.
#ifndef HYT_PPR_QUAD_INFLIGHT
#define HYT_PPR_QUAD_INFLIGHT 4
#endif
constexpr int kQuadInFlight = HYT_PPR_QUAD_INFLIGHT;  // edges loaded per thread before any is added

__device__ __forceinline__ void row_quad_sum(const uint32_t *__restrict__ in_src,
                                             const uint32_t *__restrict__ hot_vertex, const float *__restrict__ c,
                                             uint64_t b, uint64_t e, int t, double (&acc)[4]) {
    const int slot = t >> 1, h = t & 1;
    const float4 *c4 = reinterpret_cast<const float4 *>(c);
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = 0.0;
    for (uint64_t i0 = b + slot; i0 < e; i0 += 16 * kQuadInFlight) {
        uint32_t u[kQuadInFlight];
#pragma unroll
        for (int j = 0; j < kQuadInFlight; ++j) u[j] = (i0 + 16 * j < e) ? __ldcs(in_src + i0 + 16 * j) : 0u;
#pragma unroll
        for (int j = 0; j < kQuadInFlight; ++j)
            if (u[j] & kHotTag) u[j] = hot_vertex[u[j] & ~kHotTag];
        float4 v[kQuadInFlight];
#pragma unroll
        for (int j = 0; j < kQuadInFlight; ++j)
            v[j] = (i0 + 16 * j < e) ? c4[uint64_t(u[j]) * 2 + h] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < kQuadInFlight; ++j) {
            if (i0 + 16 * j < e) {
                acc[0] += double(v[j].x);
                acc[1] += double(v[j].y);
                acc[2] += double(v[j].z);
                acc[3] += double(v[j].w);
            }
        }
    }
#pragma unroll
    for (int o = 2; o < 32; o <<= 1)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
}

struct LaneParams {
    uint32_t source[kLanes];   // internal ids; lanes >= k unused
    uint32_t active;           // bit l: lane l still iterates
    double d;                  // damping
};

// The iteration's per-lane dangling mass (dm[8], summed once per
// iteration by ppr8_lane_sums_kernel), into shared memory.
__device__ __forceinline__ void lane_dangling(const double *__restrict__ dm, double *s_dm) {
    if (threadIdx.x < kLanes) s_dm[threadIdx.x] = dm[threadIdx.x];
    __syncthreads();
}

// Fixed-order per-lane sums of per-block partials: out[l] = sum over
// a[i][l] (i < na), b[i][l] (i < nb) and w[i][l] (i < nw).  One block of kSumThreads: thread t
// sums group t / 8 (partials g, g + G, g + 2G, ...; G = kSumThreads / 8),
// then thread l < 8 adds the G group sums in order.  Every thread holds a
// few dependent adds instead of one thread walking all partials (one L2
// round trip per partial).
constexpr int kSumThreads = 1024;

__global__ void __launch_bounds__(kSumThreads) ppr8_lane_sums_kernel(const double *__restrict__ a, int na,
                                                                     const double *__restrict__ b, int nb,
                                                                     const double *__restrict__ w, int nw,
                                                                     double *__restrict__ out) {
    constexpr int kGroups = kSumThreads / kLanes;
    __shared__ double s[kGroups][kLanes];
    const int l = threadIdx.x & (kLanes - 1), g = threadIdx.x / kLanes;
    double x = 0.0;
    for (int i = g; i < na; i += kGroups) x += a[size_t(i) * kLanes + l];
    for (int i = g; i < nb; i += kGroups) x += b[size_t(i) * kLanes + l];
    for (int i = g; i < nw; i += kGroups) x += w[size_t(i) * kLanes + l];
    s[g][l] = x;
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double r = 0.0;
        for (int j = 0; j < kGroups; ++j) r += s[j][threadIdx.x];
        out[threadIdx.x] = r;
    }
}

__device__ __forceinline__ float lane_next(uint64_t v, int lane, double sum, const LaneParams &p, const double *s_dm,
                                           float cur) {
    if (!((p.active >> lane) & 1u)) return cur;
    double nx = p.d * sum;
    uint32_t src = 0xFFFFFFFFu;  // p.source[lane] without a local-memory copy of p
#pragma unroll
    for (int l = 0; l < kLanes; ++l)
        if (l == lane) src = p.source[l];
    if (v == src) nx += (1.0 - p.d) + p.d * s_dm[lane];
    return float(nx);
}

// Short rows (fewer than kWideRow in-edges), 16 per warp: threads 2q and
// 2q + 1 take row v0 + q, queries 0-3 and 4-7 (one 16-byte contribution
// load per in-edge each), and add the row's in-edges in edge order, 4
// loaded before any is added.  Each thread then writes its row's four
// values; per-block residual partials per query in a fixed order.  Wider
// rows go to ppr8_wide_kernel, long rows to the chunk kernels.
constexpr uint32_t kWideRow = 32;
constexpr int kRowThreads = 256;

__global__ void __launch_bounds__(kRowThreads) ppr8_rows_kernel(
    const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_src, const uint32_t *__restrict__ hot_vertex,
    const float *__restrict__ c, const float *__restrict__ x, uint64_t V, uint64_t long_from, LaneParams p,
    const double *__restrict__ dpart, float *__restrict__ nxt, double *__restrict__ rpart) {
    __shared__ double s_dm[kLanes];
    __shared__ double s_res[kLanes][kRowThreads / 32];
    lane_dangling(dpart, s_dm);
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5, q = t >> 1, h = t & 1;
    const float4 *c4 = reinterpret_cast<const float4 *>(c);
    const uint64_t warps = uint64_t(gridDim.x) * (kRowThreads / 32);
    double res[4] = {0.0, 0.0, 0.0, 0.0};  // queries 4h .. 4h + 3
    for (uint64_t v0 = ((blockIdx.x * uint64_t(kRowThreads) + threadIdx.x) >> 5) * 16; v0 < V; v0 += warps * 16) {
        const uint64_t v = v0 + q;
        uint64_t b = 0, e = 0;
        if (v < V) {
            b = in_off[v];
            e = in_off[v + 1];
        }
        const uint64_t deg = e - b;
        // wide rows: ppr8_wide_kernel; long rows: the chunk kernels
        const bool mine = v < V && deg < kWideRow && deg < long_from;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (mine) {
            for (uint64_t i0 = b; i0 < e; i0 += 4) {
                uint32_t u[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) u[j] = (i0 + j < e) ? __ldcs(in_src + i0 + j) : 0u;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (u[j] & kHotTag) u[j] = hot_vertex[u[j] & ~kHotTag];
                float4 cv[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    cv[j] = (i0 + j < e) ? c4[uint64_t(u[j]) * 2 + h] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (i0 + j < e) {
                        acc[0] += double(cv[j].x);
                        acc[1] += double(cv[j].y);
                        acc[2] += double(cv[j].z);
                        acc[3] += double(cv[j].w);
                    }
                }
            }
        }
        if (mine) {
            const float4 cur = reinterpret_cast<const float4 *>(x)[v * 2 + h];
            const float cv[4] = {cur.x, cur.y, cur.z, cur.w};
            float nx[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                nx[k] = lane_next(v, 4 * h + k, acc[k], p, s_dm, cv[k]);
                res[k] += fabs(double(nx[k]) - double(cv[k]));
            }
            reinterpret_cast<float4 *>(nxt)[v * 2 + h] = make_float4(nx[0], nx[1], nx[2], nx[3]);
        }
    }
    // fixed-order residual partials: the 16 row slots of the warp, then warps
#pragma unroll
    for (int o = 2; o < 32; o <<= 1)
#pragma unroll
        for (int k = 0; k < 4; ++k) res[k] += __shfl_xor_sync(0xffffffffu, res[k], o);
    if (t < 2)
#pragma unroll
        for (int k = 0; k < 4; ++k) s_res[4 * t + k][warp] = res[k];
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double a = 0.0;
        for (int w = 0; w < kRowThreads / 32; ++w) a += s_res[threadIdx.x][w];
        rpart[blockIdx.x * kLanes + threadIdx.x] = a;
    }
}

// Rows of kWideRow or more in-edges below the long-row threshold (the
// graph's list `wide`), one per warp across the whole grid: hub order puts
// them together at the front of the vertex range, where warps that took
// them 16 at a time in the rows pass held up its end.  The whole warp sums
// a row (row_quad_sum); threads 0 and 1 write queries 0-3 and 4-7.
__global__ void __launch_bounds__(kRowThreads) ppr8_wide_kernel(
    const uint32_t *__restrict__ wide, uint64_t num_wide, const uint64_t *__restrict__ in_off,
    const uint32_t *__restrict__ in_src, const uint32_t *__restrict__ hot_vertex, const float *__restrict__ c,
    const float *__restrict__ x, LaneParams p, const double *__restrict__ dm, float *__restrict__ nxt,
    double *__restrict__ wpart) {
    __shared__ double s_dm[kLanes];
    __shared__ double s_res[kLanes][kRowThreads / 32];
    lane_dangling(dm, s_dm);
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t warps = uint64_t(gridDim.x) * (kRowThreads / 32);
    double res[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint64_t i = (blockIdx.x * uint64_t(kRowThreads) + threadIdx.x) >> 5; i < num_wide; i += warps) {
        const uint64_t v = wide[i];
        double sum[4];
        row_quad_sum(in_src, hot_vertex, c, in_off[v], in_off[v + 1], t, sum);  // queries 4h .. 4h + 3
        if (t < 2) {
            const float4 cur = reinterpret_cast<const float4 *>(x)[v * 2 + t];
            const float cv[4] = {cur.x, cur.y, cur.z, cur.w};
            float nx[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                nx[q] = lane_next(v, 4 * t + q, sum[q], p, s_dm, cv[q]);
                res[q] += fabs(double(nx[q]) - double(cv[q]));
            }
            reinterpret_cast<float4 *>(nxt)[v * 2 + t] = make_float4(nx[0], nx[1], nx[2], nx[3]);
        }
    }
    if (t < 2)
#pragma unroll
        for (int q = 0; q < 4; ++q) s_res[4 * t + q][warp] = res[q];
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double a = 0.0;
        for (int w = 0; w < kRowThreads / 32; ++w) a += s_res[threadIdx.x][w];
        wpart[blockIdx.x * kLanes + threadIdx.x] = a;
    }
}

// flags[v] = 1 for rows with kWideRow <= in-degree < long_from.
__global__ void ppr8_wide_flags_kernel(const uint64_t *__restrict__ in_off, uint64_t V, uint64_t long_from,
                                       uint8_t *__restrict__ flags) {
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t d = in_off[v + 1] - in_off[v];
        flags[v] = (d >= kWideRow && d < long_from) ? 1 : 0;
    }
}

// One warp per piece of a long-row chunk (each chunk cut into `pieces`
// equal pieces, so that graphs with few chunks still fill the GPU):
// per-lane partial sums, stored at (chunk * pieces + piece).
__global__ void ppr8_chunks_kernel(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_src,
                                   const uint32_t *__restrict__ hot_vertex, const float *__restrict__ c,
                                   const LongRow *__restrict__ long_rows, const uint2 *__restrict__ tasks,
                                   uint64_t num_tasks, uint32_t pieces, double *__restrict__ chunk_sum) {
    const int t = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    const uint64_t piece_edges = (kLongChunk + pieces - 1) / pieces;
    for (uint64_t k = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; k < num_tasks * pieces; k += warps) {
        const uint64_t ci = k / pieces, pc = k % pieces;
        const uint2 task = tasks[ci];
        const LongRow lr = long_rows[task.x];
        const uint64_t cb = in_off[lr.row] + uint64_t(task.y) * kLongChunk;
        const uint64_t ce = min(cb + kLongChunk, in_off[lr.row + 1]);
        const uint64_t b = min(cb + pc * piece_edges, ce), e = min(b + piece_edges, ce);
        double sum[4];
        row_quad_sum(in_src, hot_vertex, c, b, e, t, sum);
        if (t < 2)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                chunk_sum[((uint64_t(lr.first_chunk) + task.y) * pieces + pc) * kLanes + 4 * t + q] = sum[q];
    }
}

// One warp per long row: chunk partials in order, next values, residual.
__global__ void ppr8_long_rows_kernel(const LongRow *__restrict__ long_rows, uint64_t num_long, uint32_t pieces,
                                      const double *__restrict__ chunk_sum, const float *__restrict__ x, LaneParams p,
                                      const double *__restrict__ dpart, float *__restrict__ nxt,
                                      double *__restrict__ rpart) {
    __shared__ double s_dm[kLanes];
    __shared__ double s_res[kLanes][8];
    lane_dangling(dpart, s_dm);
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    double res = 0.0;
    for (uint64_t i = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; i < num_long; i += warps) {
        const LongRow lr = long_rows[i];
        if (t < kLanes) {
            double sum = 0.0;
            const uint64_t first = uint64_t(lr.first_chunk) * pieces, n = uint64_t(lr.num_chunks) * pieces;
            for (uint64_t k = 0; k < n; ++k) sum += chunk_sum[(first + k) * kLanes + t];
            const uint64_t v = lr.row;
            const float cur = x[v * kLanes + t];
            const float nx = lane_next(v, t, sum, p, s_dm, cur);
            nxt[v * kLanes + t] = nx;
            res += fabs(double(nx) - double(cur));
        }
    }
    if (t < kLanes) s_res[t][warp] = res;
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double a = 0.0;
        for (int w = 0; w < 8; ++w) a += s_res[threadIdx.x][w];
        rpart[blockIdx.x * kLanes + threadIdx.x] = a;
    }
}

// ---- staged task pass (graph in HBM: pull task descriptors) -----------------
//
// The pull tasks (stage.cuh) replace the one-warp-per-row pass: a warp
// stages each tile's (or chunk piece's) source ids in shared memory one
// unit ahead, then
//   tile rows  -- 4 rows at a time, thread t owning row rb + t / 8 and lane
//                 t % 8: the 8 threads of a row read one id (a shared-memory
//                 broadcast) and one 32-byte contribution sector per
//                 in-edge, kUnroll edges in flight per thread; rows of >= 64
//                 in-edges are taken by the whole warp in a 4-slot layout
//                 (thread t: edge slot t / 8, lane t % 8);
//   chunks     -- the same 4-slot layout over the chunk's edges, one FP64
//                 partial per chunk and lane (summed by
//                 ppr8_long_rows_kernel).
// Every sum is FP64 in a fixed edge order and the thread layout does not
// depend on the lane count, so a query's bits do not depend on its
// companions.  Residual partials are per block over a static task
// assignment (fixed for a fixed grid).
constexpr int kTaskThreads = stage::kStageThreads;
constexpr int kUnroll = 8;

// Sum over in-edges [b, e) of c[u][lane] from staged ids, thread t taking
// edge slot t / 8 (4 slots) and lane t % 8; complete in every thread.
__device__ __forceinline__ double staged_lane_sum(const uint32_t *slot, uint64_t a0, const uint32_t *s_hot,
                                                  const float *__restrict__ c, uint64_t b, uint64_t e, int t) {
    const int sl = t >> 3, lane = t & 7;
    double acc = 0.0;
    for (uint64_t i = b + sl; i < e; i += 4 * kUnroll) {
        float g[kUnroll];
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) {
            const uint64_t x = i + 4 * q;
            uint32_t u = x < e ? slot[x - a0] : 0u;
            if (u & kHotTag) u = s_hot[u & ~kHotTag];
            g[q] = x < e ? __ldcg(c + uint64_t(u) * kLanes + lane) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) acc += double(g[q]);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    return acc;
}

__global__ void __launch_bounds__(kTaskThreads, 1)
    ppr8_tasks_kernel(const uint4 *__restrict__ tasks, uint64_t num_tasks, const uint64_t *__restrict__ in_off,
                      const uint32_t *__restrict__ in_src, const uint32_t *__restrict__ hot_vertex, uint32_t num_hot,
                      const LongRow *__restrict__ long_rows, const float *__restrict__ c,
                      const float *__restrict__ x, LaneParams p, const double *__restrict__ dpart,
                      float *__restrict__ nxt, double *__restrict__ chunk_sum, double *__restrict__ rpart,
                      uint32_t *__restrict__ error) {
    extern __shared__ __align__(128) unsigned char s_stage[];
    __shared__ double s_dm[kLanes];
    __shared__ double s_res[kLanes][kTaskThreads / 32];
    lane_dangling(dpart, s_dm);
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const stage::WarpStage ws = stage::warp_stage(s_stage, warp, t);
    uint32_t *s_hot = reinterpret_cast<uint32_t *>(s_stage + stage::kStageBytes);
    for (uint32_t i = threadIdx.x; i < num_hot; i += blockDim.x) s_hot[i] = hot_vertex[i];
    __syncthreads();
    const uint64_t nwarps = uint64_t(gridDim.x) * (kTaskThreads / 32);
    const int lane = t & 7, rsub = t >> 3;
    double res = 0.0;  // this thread's lane, rows of this warp's tasks in task order
    double acc = 0.0;  // running chunk sum
    const bool ok = stage::stage_pipeline(
        tasks, in_src, uint64_t(blockIdx.x) * (kTaskThreads / 32) + warp, nwarps, num_tasks, ws, t,
        [&](uint4 d, uint64_t, uint32_t j, uint32_t nu, uint32_t *slot, uint64_t a0) {
            if (task_is_chunk(d)) {
                const stage::Unit u = stage::unit_of(d, j);
                if (j == 0) acc = 0.0;
                // the 4-slot layout over the whole chunk: slot sl takes
                // edges lo + sl, lo + sl + 4, ... of every piece in order
                const int sl = t >> 3;
                for (uint64_t i = u.lo + sl; i < u.hi; i += 4 * kUnroll) {
                    float g[kUnroll];
#pragma unroll
                    for (int q = 0; q < kUnroll; ++q) {
                        const uint64_t xx = i + 4 * q;
                        uint32_t v = xx < u.hi ? slot[xx - a0] : 0u;
                        if (v & kHotTag) v = s_hot[v & ~kHotTag];
                        g[q] = xx < u.hi ? __ldcg(c + uint64_t(v) * kLanes + lane) : 0.0f;
                    }
#pragma unroll
                    for (int q = 0; q < kUnroll; ++q) acc += double(g[q]);
                }
                if (j + 1 < nu) return;
                double sum = acc;
                sum += __shfl_xor_sync(0xffffffffu, sum, 8);
                sum += __shfl_xor_sync(0xffffffffu, sum, 16);
                if (t < kLanes) chunk_sum[(uint64_t(long_rows[d.z].first_chunk) + d.w) * kLanes + t] = sum;
                return;
            }
            const uint32_t r0 = d.z, rl = d.w;
            for (uint32_t rb = r0; rb < rl; rb += 4) {
                const uint32_t r = rb + rsub;
                const bool active = r < rl;
                const uint64_t lo = active ? in_off[r] : 0, hi = active ? in_off[r + 1] : 0;
                const bool small = active && hi - lo < 64;
                double sum = 0.0;
                if (small) {
                    for (uint64_t i = lo; i < hi; i += kUnroll) {
                        float g[kUnroll];
#pragma unroll
                        for (int q = 0; q < kUnroll; ++q) {
                            const uint64_t xx = i + q;
                            uint32_t v = xx < hi ? slot[xx - a0] : 0u;
                            if (v & kHotTag) v = s_hot[v & ~kHotTag];
                            g[q] = xx < hi ? __ldcg(c + uint64_t(v) * kLanes + lane) : 0.0f;
                        }
#pragma unroll
                        for (int q = 0; q < kUnroll; ++q) sum += double(g[q]);
                    }
                }
                // rows of >= 64 in-edges: the whole warp, one row at a time
                uint32_t big = __ballot_sync(0xffffffffu, active && !small) & 0x01010101u;
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, hi, src);
                    const double s2 = staged_lane_sum(slot, a0, s_hot, c, bb, ee, t);
                    if ((src >> 3) == rsub) sum = s2;
                }
                if (active) {
                    const float cur = x[uint64_t(r) * kLanes + lane];
                    const float nx = lane_next(r, lane, sum, p, s_dm, cur);
                    nxt[uint64_t(r) * kLanes + lane] = nx;
                    res += fabs(double(nx) - double(cur));
                }
            }
        });
    if (!ok) atomicExch(error, 1u);
    // per-lane residual: the warp's 4 row slots, then the block's warps in order
    res += __shfl_xor_sync(0xffffffffu, res, 8);
    res += __shfl_xor_sync(0xffffffffu, res, 16);
    if (t < kLanes) s_res[t][warp] = res;
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double a = 0.0;
        for (int w = 0; w < kTaskThreads / 32; ++w) a += s_res[threadIdx.x][w];
        rpart[blockIdx.x * kLanes + threadIdx.x] = a;
    }
}

__global__ void ppr8_init_kernel(float *__restrict__ x, uint64_t V, LaneParams p, int k) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < V * kLanes;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const int lane = int(i & 7);
        const uint64_t v = i >> 3;
        x[i] = (lane < k && v == p.source[lane]) ? 1.0f : 0.0f;
    }
}

__global__ void ppr8_lane_kernel(const float *__restrict__ x, uint64_t V, int lane, float *__restrict__ out) {
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x)
        out[v] = x[v * kLanes + lane];
}

unsigned grid_sm(unsigned per_sm) { return static_cast<unsigned>(sm_count()) * per_sm; }

}  // namespace

void ppr_multi(GraphImpl &g, const uint32_t *sources, uint32_t k, float restart, float tolerance, uint32_t max_iter,
               float *out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    if (k == 0 || k > kLanes) fail(HYT_E_INVALID, "hyt_ppr_multi takes 1 to 8 sources");
    if (!sources) fail(HYT_E_INVALID, "sources is NULL");
    if (!(restart > 0.0f && restart <= 1.0f)) fail(HYT_E_INVALID, "personalized PageRank restart must be in (0, 1]");
    if (!(tolerance > 0.0f) || !std::isfinite(tolerance))
        fail(HYT_E_INVALID, "personalized PageRank tolerance must be finite and positive");
    if (max_iter == 0) fail(HYT_E_INVALID, "personalized PageRank max_iterations must be greater than zero");
    const uint64_t V = g.V;
    for (uint32_t l = 0; l < k; ++l)
        if (sources[l] >= V) fail(HYT_E_INVALID, "personalized PageRank source vertex is out of range");
    if (stats) std::memset(stats, 0, sizeof(hyt_run_stats) * k);
    HYT_CUDA(cudaSetDevice(g.device));
    cudaStream_t s = g.stream;
    LaneParams p{};
    for (uint32_t l = 0; l < kLanes; ++l) p.source[l] = l < k ? graph_vertex(g, sources[l], s) : 0xFFFFFFFFu;
    p.active = (1u << k) - 1u;
    p.d = 1.0 - double(restart);
    // staged task pass when the graph carries task descriptors (in HBM)
    const bool staged = g.pull_tasks.get() && g.tile_cost <= kStageTileMax &&
                        stage::staged_shared_bytes(g.num_hot) + 4096 <= kPRSmemMax;
    const unsigned smem = static_cast<unsigned>(stage::staged_shared_bytes(g.num_hot));
    if (staged) {
        // the kernel's static shared memory counts against the same
        // per-block limit, so ask for exactly what this launch uses
        static unsigned attr = 0;
        if (smem > attr) {
            HYT_CUDA(cudaFuncSetAttribute(ppr8_tasks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
            attr = smem;
        }
    }
    // one persistent wave of the rows pass (its partials are summed in block order)
    static int rows_per_sm = 0;
    if (!staged && rows_per_sm == 0) {
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rows_per_sm, ppr8_rows_kernel, kRowThreads, 0));
        rows_per_sm = std::max(rows_per_sm, 1);
    }
    const unsigned rows_grid = staged ? grid_sm(1) : grid_sm(rows_per_sm);
    const uint64_t chunks = g.num_long ? g.num_chunks : 0;
    const uint64_t long_from = g.num_long ? g.tile_cost : ~uint64_t(0);
    const unsigned long_grid = g.num_long ? grid_for(g.num_long * 32, 256) : 0;
    // chunks cut into pieces until there are enough warp tasks to fill the
    // GPU (a function of the graph alone, so results do not depend on it)
    uint32_t pieces = 1;
    if (!staged)
        while (pieces < 8 && chunks * pieces < 16384) pieces *= 2;
    // the graph's wide rows (once per graph)
    if (!staged && !g.ppr_wide_ready) {
        Scratch<uint8_t> flags(V, s);
        ppr8_wide_flags_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.in_offsets.get(), V, long_from, flags.get());
        HYT_CUDA(cudaGetLastError());
        g.ppr_wide.allocate(std::max<uint64_t>(V, 1));
        g.ppr_wide_n = prims::select_flagged_index(flags.get(), g.ppr_wide.get(), V, s);
        g.ppr_wide_ready = true;
    }
    const uint64_t num_wide = staged ? 0 : g.ppr_wide_n;
    static int wide_per_sm = 0;
    if (wide_per_sm == 0) {
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wide_per_sm, ppr8_wide_kernel, kRowThreads, 0));
        wide_per_sm = std::max(wide_per_sm, 1);
    }
    const unsigned wide_grid = num_wide ? grid_sm(wide_per_sm) : 0;
    Scratch<float> xa(V * kLanes, s), xb(V * kLanes, s), c(V * kLanes, s);
    Scratch<double> dpart(uint64_t(kPartBlocks) * kLanes, s), rpart(uint64_t(rows_grid) * kLanes, s),
        lpart(uint64_t(std::max(long_grid, 1u)) * kLanes, s), chunk_sum(std::max<uint64_t>(chunks * pieces, 1) * kLanes, s),
        residual(kLanes, s), dm(kLanes, s), wpart(uint64_t(std::max(wide_grid, 1u)) * kLanes, s);
    Scratch<uint32_t> err(1, s);
    HYT_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(uint32_t), s));
    double *h_res = reinterpret_cast<double *>(g.host_scratch.ptr);  // 64 pinned bytes
    float *x = xa.get(), *nx = xb.get();
    ppr8_init_kernel<<<grid_sm(8), 256, 0, s>>>(x, V, p, int(k));
    HYT_CUDA(cudaGetLastError());
    std::vector<uint32_t> iters(k, 0);
    std::vector<double> last(k, 0.0);
    EventTimer timer;
    timer.start(s);
    uint64_t launches = 1;
    for (uint32_t it = 0; it < max_iter && p.active; ++it) {
        ppr8_prep_kernel<<<kPartBlocks, 256, 0, s>>>(g.out_degree.get(), x, V, c.get(), dpart.get());
        ppr8_lane_sums_kernel<<<1, kSumThreads, 0, s>>>(dpart.get(), kPartBlocks, nullptr, 0, nullptr, 0, dm.get());
        launches += 3;
        if (staged) {
            ppr8_tasks_kernel<<<rows_grid, kTaskThreads, smem, s>>>(
                g.pull_tasks.get(), g.num_chunks + g.num_tiles, g.in_offsets.get(), g.in_sources.get(),
                g.hot_vertex.get(), g.num_hot, g.long_rows.get(), c.get(), x, p, dm.get(), nx, chunk_sum.get(),
                rpart.get(), err.get());
            if (chunks) {
                ppr8_long_rows_kernel<<<long_grid, 256, 0, s>>>(g.long_rows.get(), g.num_long, 1u, chunk_sum.get(),
                                                                x, p, dm.get(), nx, lpart.get());
                ++launches;
            }
        } else {
            ppr8_rows_kernel<<<rows_grid, kRowThreads, 0, s>>>(g.in_offsets.get(), g.in_sources.get(),
                                                               g.hot_vertex.get(), c.get(), x, V, long_from, p,
                                                               dm.get(), nx, rpart.get());
            if (num_wide) {
                ppr8_wide_kernel<<<wide_grid, kRowThreads, 0, s>>>(g.ppr_wide.get(), num_wide, g.in_offsets.get(),
                                                                   g.in_sources.get(), g.hot_vertex.get(), c.get(), x,
                                                                   p, dm.get(), nx, wpart.get());
                ++launches;
            }
        }
        if (chunks && !staged) {
            ppr8_chunks_kernel<<<grid_sm(8), 256, 0, s>>>(g.in_offsets.get(), g.in_sources.get(), g.hot_vertex.get(),
                                                          c.get(), g.long_rows.get(), g.chunk_tasks.get(), chunks,
                                                          pieces, chunk_sum.get());
            ppr8_long_rows_kernel<<<long_grid, 256, 0, s>>>(g.long_rows.get(), g.num_long, pieces, chunk_sum.get(), x,
                                                            p, dm.get(), nx, lpart.get());
            launches += 2;
        }
        ppr8_lane_sums_kernel<<<1, kSumThreads, 0, s>>>(rpart.get(), int(rows_grid), lpart.get(),
                                                        int(chunks ? long_grid : 0), wpart.get(), int(wide_grid),
                                                        residual.get());
        ++launches;
        HYT_CUDA(cudaGetLastError());
        HYT_CUDA(cudaMemcpyAsync(h_res, residual.get(), kLanes * 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        std::swap(x, nx);
        for (uint32_t l = 0; l < k; ++l) {
            if (!((p.active >> l) & 1u)) continue;
            iters[l] = it + 1;
            last[l] = h_res[l];
            if (h_res[l] <= double(tolerance)) p.active &= ~(1u << l);
        }
    }
    timer.stop(s);
    const double ms = timer.ms();
    uint32_t h_err = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(h_err), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (h_err) fail(HYT_E_TIMEOUT, "hyt_ppr_multi: a bounded wait for a staged copy ran out");
    if (out) {
        Scratch<float> lane(V, s);
        for (uint32_t l = 0; l < k; ++l) {
            ppr8_lane_kernel<<<grid_for(V, 256), 256, 0, s>>>(x, V, int(l), lane.get());
            HYT_CUDA(cudaGetLastError());
            graph_emit(g, out + uint64_t(l) * V, lane.get(), s);
        }
    }
    HYT_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        for (uint32_t l = 0; l < k; ++l) {
            stats[l].iterations = iters[l];
            stats[l].converged = ((p.active >> l) & 1u) ? 0u : 1u;
            stats[l].residual = last[l];
            stats[l].device_ms = ms;
            stats[l].total_launches = static_cast<uint32_t>(launches);
            stats[l].edges_processed = g.E * iters[l];
            stats[l].vertices_processed = V * iters[l];
        }
        // one pass for all lanes: source id + one 32-byte contribution sector
        // per in-edge; per vertex: offsets, the 8 lanes read and written,
        // contributions written
        const uint64_t iterations = *std::max_element(iters.begin(), iters.end());
        stats[0].algorithmic_bytes = iterations * (36 * g.E + (8 + 32 + 32 + 32 + 4) * V);
    }
}

}  // namespace hyt
