// PageRank and personalized PageRank: synchronous (Jacobi) pull over the CSC.
//
// Semantics follow the reference CPU solver (src/algorithms/pagerank.cpp:
// 89-163): x_0 = 1/n; each step
//     x'[v] = (1-d)/n + d * dangling / n + d * sum_{u->v} x[u] / deg(u)
// with dangling = sum of x over out-degree-0 vertices, residual = L1 change,
// stop when residual <= tolerance or after max_iterations.  Per-edge
// contributions x[u]/deg(u) are formed once per vertex in the producing
// step (the reference divides per edge, same float quotient).  In-row sums
// are compensated (TwoSum/Kahan) in FP32; residual and dangling mass are
// reduced in FP64.
//
// One persistent kernel per iteration (1024 threads, one CTA per SM).  The
// work list is the graph's pull tasks, assigned to warps round-robin
// (warp w takes tasks w, w + W, ...; every task costs at most kLongChunk
// edges, so no shared counter is needed):
//   chunk tasks  -- kLongChunk-edge slices of rows with in-degree >=
//                   tile_cost; each warp writes a compensated partial, the
//                   last arriving warp of a row merges the partials in chunk
//                   order;
//   tile tasks   -- merge-path tiles of consecutive shorter rows (512
//                   units by default); the tile's contributions are
//                   gathered, 16 per lane in flight, into the warp's
//                   shared-memory slice, then summed lane-per-row (in-degree
//                   < kWarpRowDegree) or warp-per-row.  The first 32 rows'
//                   bounds, ranks and out-degrees are loaded with the
//                   gathers, and before its row phase a warp warms L2 with
//                   its next task's id lines.
// With HYT_STAGED=1 (256-unit tiles) pr_staged_kernel stages each task's
// source ids in shared memory by bulk copies (cp.async.bulk, completion on
// an mbarrier; stage.cuh) instead; on R-MAT graphs it ran slower than the
// register path.  The out-of-HBM solver, whose ids come from staging slots
// or mapped host memory, runs the register path over its partitions.
//
// Results are deterministic: every row sum has a fixed association order,
// and the FP64 residual and dangling mass are summed in a fixed slot order
// (PRSlots), independent of the grid size and of warp arrival order: each
// task stores its slot, then pr_reduce_kernel sums the slots and evaluates
// the stop rule, ending the CUDA-graph conditional while-loop when done.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "bulk.cuh"
#include "common.cuh"
#include "graph.cuh"
#include "hybrid.cuh"
#include "pagerank_core.cuh"
#include "solvers.cuh"
#include "stage.cuh"

namespace hyt {
namespace {

using namespace prc;
using namespace stage;

// Slot of long row i and of tile k in the fixed-order reduction.
__device__ __forceinline__ uint32_t long_slot(uint32_t i) { return i; }
__device__ __forceinline__ uint32_t tile_slot(const PRArgs &a, uint64_t k) {
    return a.red.num_slots - static_cast<uint32_t>(a.num_tiles) + static_cast<uint32_t>(k);
}

// Hot-source contributions of this iteration, loaded once per CTA.
__device__ __forceinline__ void load_hot(const PRArgs &a, const PRBuffers &b, float *s_hot) {
    const uint32_t nt = blockDim.x;
    for (uint32_t i0 = 0; i0 < a.num_hot; i0 += 8 * nt) {
        uint32_t hv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * nt + threadIdx.x;
            hv[k] = (i < a.num_hot) ? a.hot_vertex[i] : 0u;
        }
        float hc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) hc[k] = b.ccur[hv[k]];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * nt + threadIdx.x;
            if (i < a.num_hot) s_hot[i] = hc[k];
        }
    }
}

// ---- register path (out-of-HBM partitioned solves) ------------------------

// One launch processes chunk tasks [chunk_begin, chunk_end) and tiles
// [tile_begin, tile_end); in_src is the base of the source ids, addressed by
// global edge index (a device array, a staging slot offset by its first
// edge, or mapped host memory).  An iteration may span several launches;
// pr_reduce_kernel closes it after the last one.
struct PRRange {
    const uint32_t *in_src;
    uint64_t chunk_begin, chunk_end, tile_begin, tile_end;
    const uint4 *tasks;  // the graph's task descriptors (whole-graph launches; NULL: no prefetch)
};

__global__ void __launch_bounds__(kPRThreads, 1) pr_iterate_kernel(const PRArgs *__restrict__ args, PRRange rg) {
    extern __shared__ __align__(16) float s_dyn[];

    const PRArgs a = *args;
    const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
    if (*(volatile uint32_t *)&a.hdr->done) return;

    const PRBuffers b = buffers(a, it);
    const PRState ps = make_state(a, a.dangling[it]);
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t n_chunks = rg.chunk_end - rg.chunk_begin;
    const uint64_t total_tasks = n_chunks + (rg.tile_end - rg.tile_begin);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *s_hot = s_dyn;
    load_hot(a, b, s_hot);
    __syncthreads();
    float *sv = s_dyn + a.num_hot + warp * (2 * a.tile_cost + 8);
    const uint64_t nwarps = uint64_t(gridDim.x) * (kPRThreads / 32);

    for (uint64_t task = uint64_t(blockIdx.x) * (kPRThreads / 32) + warp; task < total_tasks; task += nwarps) {
        double res = 0.0, dang = 0.0;
        // whole-graph launches index the descriptors like their tasks
        const uint64_t next = task + nwarps;
        const uint4 nd = (rg.tasks && next < total_tasks) ? rg.tasks[next] : make_uint4(0, 0, 0, 0);
        const uint4 *pf = rg.tasks ? &nd : nullptr;
        if (task < n_chunks) {
            const uint32_t row = chunk_task<true>(a, ps, b, rg.in_src, s_hot, rg.chunk_begin + task, pol, lane, res,
                                                  dang, pf);
            if (row != ~0u) slot_store(a, long_slot(row), dev::warp_sum(res), dev::warp_sum(dang), lane);
        } else {
            const uint64_t k = rg.tile_begin + (task - n_chunks);
            tile_task<true>(a, ps, b, rg.in_src, s_hot, sv, k, pol, lane, res, dang, pf);
            slot_store(a, tile_slot(a, k), dev::warp_sum(res), dev::warp_sum(dang), lane);
        }
    }
}

// ---- staged path (graph in HBM; pipeline in stage.cuh) ---------------------

__device__ __forceinline__ void stage_failed(const PRArgs &a) {
    atomicExch(&a.hdr->error, 1u);
    atomicExch(&a.hdr->done, 1u);
    if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
}

// Gathers the contributions of staged edges [lo, hi) (ids at
// slot[x - a0]): lane l takes edges lo + 32k + l, all kUnitEdges / 32
// gathers in flight.  sink(i, value) receives edge lo + i.
template <class Sink>
__device__ __forceinline__ void gather_staged(const uint32_t *slot, uint64_t a0, uint64_t lo, uint64_t hi,
                                              const float *ccur, const float *s_hot, uint64_t pol, int lane,
                                              Sink &&sink) {
    constexpr int kB = kUnitEdges / 32;
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    const uint32_t *ids = slot + (lo - a0);
    float v[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const uint32_t i = 32 * k + lane;
        const uint32_t id = (i < n) ? ids[i] : 0u;
        v[k] = (id & kHotTag) ? s_hot[id & ~kHotTag] : dev::ld_keep(ccur + id, pol);
    }
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const uint32_t i = 32 * k + lane;
        if (i < n) sink(i, v[k]);
    }
}

__global__ void __launch_bounds__(kStageThreads, 1) pr_staged_kernel(const PRArgs *__restrict__ args) {
    extern __shared__ __align__(128) unsigned char s_stage[];
    const PRArgs a = *args;
    const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
    if (*(volatile uint32_t *)&a.hdr->done) return;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const WarpStage ws = warp_stage(s_stage, warp, lane);
    float *s_hot = reinterpret_cast<float *>(s_stage + kStageBytes);
    const PRBuffers b = buffers(a, it);
    const PRState ps = make_state(a, a.dangling[it]);
    const uint64_t pol = dev::policy_evict_last();
    load_hot(a, b, s_hot);
    __syncthreads();

    const uint64_t total = a.num_chunks + a.num_tiles;
    const uint64_t nwarps = uint64_t(gridDim.x) * kStageWarps;
    dev::CSum acc;  // running sum of the current chunk
    const bool ok = stage_pipeline(
        a.tasks, a.in_src, uint64_t(blockIdx.x) * kStageWarps + warp, nwarps, total, ws, lane,
        [&](uint4 d, uint64_t task, uint32_t j, uint32_t nu, uint32_t *slot, uint64_t a0) {
            double res = 0.0, dang = 0.0;
            if (task_is_chunk(d)) {
                const Unit u = unit_of(d, j);
                if (j == 0) acc = dev::CSum();
                gather_staged(slot, a0, u.lo, u.hi, b.ccur, s_hot, pol, lane, [&](uint32_t, float v) { acc.add(v); });
                if (j + 1 < nu) return;
                // last piece: publish the chunk's partial; the row's last
                // arriving chunk merges the partials in chunk order
                const LongRow L = a.long_rows[d.z];
                const dev::CSum w = dev::warp_reduce(acc);
                uint32_t last = 0;
                if (lane == 0) {
                    a.partial[L.first_chunk + d.w] = make_float2(w.s, w.c);
                    __threadfence();
                    const uint32_t tk = atomicAdd(&a.ticket[d.z], 1u) + 1u;
                    last = (tk % L.num_chunks == 0) ? 1u : 0u;
                }
                if (!__shfl_sync(0xffffffffu, last, 0)) return;
                __threadfence();
                dev::CSum row;
                for (uint32_t c = lane; c < L.num_chunks; c += 32) {
                    const float2 p = __ldcg(a.partial + L.first_chunk + c);
                    dev::CSum x;
                    x.s = p.x;
                    x.c = p.y;
                    row.merge(x);
                }
                row = dev::warp_reduce(row);
                if (lane == 0) finalize_row(a, ps, L.row, row.value(), b.cur, b.nxt, b.cnxt, res, dang);
                slot_store(a, long_slot(d.z), res, dang, lane);  // lane 0 finalized the row
                return;
            }
            // tile: rows [r0, rl), edges [e0, e0 + n); contributions replace
            // the ids in the slot, then rows are summed in edge order
            const uint32_t r0 = d.z, rl = d.w;
            const uint64_t e0 = task_first_edge(d), e1 = e0 + task_edges(d);
            float *vals = reinterpret_cast<float *>(slot);
            const uint32_t r = r0 + lane;
            const uint64_t lo0 = (r < rl) ? a.in_off[r] : 0, hi0 = (r < rl) ? a.in_off[r + 1] : 0;  // in flight
            gather_staged(slot, a0, e0, e1, b.ccur, s_hot, pol, lane,
                          [&](uint32_t i, float v) { vals[e0 - a0 + i] = v; });
            __syncwarp();
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t rr = rb + lane;
                const bool active = rr < rl;
                const uint64_t lo = (rb == r0) ? lo0 : (active ? a.in_off[rr] : 0);
                const uint64_t hi = (rb == r0) ? hi0 : (active ? a.in_off[rr + 1] : 0);
                if (active && hi - lo < kWarpRowDegree) {
                    dev::CSum s;
                    for (uint64_t x = lo; x < hi; ++x) s.add(vals[x - a0]);
                    finalize_row(a, ps, rr, s.value(), b.cur, b.nxt, b.cnxt, res, dang);
                }
                uint32_t big = __ballot_sync(0xffffffffu, active && (hi - lo >= kWarpRowDegree));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, lo, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, hi, src);
                    dev::CSum s;
                    for (uint64_t x = bb + lane; x < ee; x += 32) s.add(vals[x - a0]);
                    s = dev::warp_reduce(s);
                    if (lane == 0) finalize_row(a, ps, rb + src, s.value(), b.cur, b.nxt, b.cnxt, res, dang);
                }
            }
            slot_store(a, tile_slot(a, task - a.num_chunks), dev::warp_sum(res), dev::warp_sum(dang), lane);
        });
    if (!ok) stage_failed(a);
}

// Closes an iteration: block b sums slot groups b, b + grid, ... (thread t
// takes slots t, t + 256, ... of the group, then a fixed block tree); the
// last block to finish sums the group sums in group order, then applies
// the stop rule (ending the CUDA-graph loop when the solve is done).
constexpr int kReduceThreads = 256;

__global__ void __launch_bounds__(kReduceThreads) pr_reduce_kernel(const PRArgs *__restrict__ args) {
    __shared__ double s_red[32];
    __shared__ uint32_t s_last;
    const PRArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done) return;
    const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
    const PRSlots &R = a.red;
    for (uint32_t g = blockIdx.x; g < R.num_groups; g += gridDim.x) {
        const uint32_t b = g * kSlotGroup, n = min(kSlotGroup, R.num_slots - b);
        double r = 0.0, d = 0.0;
        for (uint32_t i = threadIdx.x; i < n; i += kReduceThreads) {
            const double2 x = __ldcg(R.slot + b + i);
            r += x.x;
            d += x.y;
        }
        r = dev::block_sum(r, s_red);
        __syncthreads();
        d = dev::block_sum(d, s_red);
        if (threadIdx.x == 0) R.group_sum[g] = make_double2(r, d);
        __syncthreads();
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(R.blocks_done, 1u) + 1u == (it + 1) * gridDim.x) ? 1u : 0u;
    __syncthreads();
    if (!s_last || threadIdx.x >= 32) return;
    __threadfence();
    double r = 0.0, d = 0.0;
    for (uint32_t g = threadIdx.x; g < R.num_groups; g += 32) {
        const double2 x = __ldcg(R.group_sum + g);
        r += x.x;
        d += x.y;
    }
    r = dev::warp_sum(r);
    d = dev::warp_sum(d);
    if (threadIdx.x == 0) close_iteration(a, it, r, d);
}

// Initial ranks and contributions; the initial dangling mass is summed in a
// fixed order: per kInitChunk-vertex chunk (a fixed thread mapping and block
// tree), then the chunk partials in chunk order by the last block.
constexpr uint32_t kInitChunk = 4096;
constexpr int kInitThreads = 256;

__global__ void __launch_bounds__(kInitThreads) pr_init_kernel(const PRArgs *__restrict__ args, double *part,
                                                               uint32_t *count) {
    __shared__ double s_red[32];
    __shared__ uint32_t s_last;
    const PRArgs a = *args;
    const uint32_t V = a.V;
    const uint32_t nchunks = (V + kInitChunk - 1) / kInitChunk;
    const float r0_uniform = __fdiv_rn(1.0f, static_cast<float>(V));
    for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        double dang = 0.0;
        const uint32_t end = min(V, (c + 1) * kInitChunk);
        for (uint32_t v = c * kInitChunk + threadIdx.x; v < end; v += kInitThreads) {
            const float r0 = a.personalized ? (v == a.source ? 1.0f : 0.0f) : r0_uniform;
            a.rank[0][v] = r0;
            const uint32_t od = a.out_deg[v];
            a.contrib[0][v] = od ? __fdiv_rn(r0, static_cast<float>(od)) : 0.0f;
            if (od == 0) dang += r0;
        }
        const double bsum = dev::block_sum(dang, s_red);
        if (threadIdx.x == 0) part[c] = bsum;
        __syncthreads();
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(count, 1u) + 1u == gridDim.x) ? 1u : 0u;
    __syncthreads();
    if (!s_last || threadIdx.x >= 32) return;
    __threadfence();
    double d = 0.0;
    for (uint32_t i = threadIdx.x; i < nchunks; i += 32) d += __ldcg(part + i);
    d = dev::warp_sum(d);
    if (threadIdx.x == 0) a.dangling[0] = d;
}

// Persistent grid of the iteration kernels: one CTA per SM, or HYT_PR_GRID
// CTAs (results do not depend on it).
int pr_occupancy_grid() {
    static int grid = 0;
    if (grid == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaFuncSetAttribute(pr_iterate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaFuncSetAttribute(pr_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_iterate_kernel, kPRThreads, kPRSmemMax));
        grid = sm_count() * std::max(per_sm, 1);
        if (const char *e = std::getenv("HYT_PR_GRID")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v > 0 && v <= 65535) grid = static_cast<int>(v);
        }
    }
    return grid;
}

// Grid of the staged kernel: one CTA per SM, or HYT_PR_GRID CTAs.
int pr_staged_grid() {
    static int grid = 0;
    if (grid == 0) {
        grid = sm_count();
        if (const char *e = std::getenv("HYT_PR_GRID")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v > 0 && v <= 65535) grid = static_cast<int>(v);
        }
    }
    return grid;
}

// In-HBM solves use the staged kernel when it was asked for (HYT_STAGED=1)
// and the graph's tiles fit a staging slot.
bool pr_use_staged(const GraphImpl &g) {
    return stage::staged_requested() && g.tile_cost <= kStageTileMax && g.pull_tasks.get() &&
           staged_shared_bytes(g.num_hot) <= kPRSmemMax;
}

}  // namespace

// Shared by PageRank and personalized PageRank.
// Workspaces, device state layout and kernel arguments of one solve.
struct PRSolveState {
    PRArgs a;
    PRArgs *d_args;
    PRHeader *hdr;
    size_t zero_bytes;
    double *init_part;
    uint32_t *init_count;
};

// pr_state layout: args | header | residual[max_iter] | dangling[max_iter+1]
// | init partials | init counter | reduce-blocks counter | (16-byte aligned)
// group sums | slots.  Everything from the header through the counters is
// cleared at the start of a solve.
static PRSolveState pr_prepare(GraphImpl &g, bool personalized, uint32_t source, float damping, float tolerance,
                               uint32_t max_iter) {
    const uint64_t V = g.V;
    // Workspaces (grown on demand, kept in the handle).
    for (int i = 0; i < 2; ++i) {
        if (g.rank[i].count < V) g.rank[i].allocate(V);
        if (g.contrib[i].count < V) g.contrib[i].allocate(V);
    }
    if (g.partial.count < 2 * std::max<uint64_t>(g.num_chunks, 1)) g.partial.allocate(2 * std::max<uint64_t>(g.num_chunks, 1));
    if (g.ticket.count < std::max<uint64_t>(g.num_long, 1)) g.ticket.allocate(std::max<uint64_t>(g.num_long, 1));
    const uint64_t num_slots = g.num_long + g.num_tiles;
    if (num_slots > 0xFFFFFFFFull) fail(HYT_E_UNSUPPORTED, "PageRank: too many pull tasks for one graph");
    const uint64_t num_groups = (num_slots + kSlotGroup - 1) / kSlotGroup;
    const uint64_t init_chunks = (V + kInitChunk - 1) / kInitChunk;
    auto up16 = [](size_t x) { return (x + 15) & ~size_t(15); };  // double2 needs 16-byte alignment
    const size_t args_bytes = (sizeof(PRArgs) + 255) & ~size_t(255);
    const size_t head = sizeof(PRHeader) + size_t(max_iter) * sizeof(double) + size_t(max_iter + 1) * sizeof(double) +
                        size_t(init_chunks) * sizeof(double) + 2 * sizeof(uint32_t);
    const size_t sb = args_bytes + up16(head) + size_t(num_groups + num_slots) * sizeof(double2) + 64;
    if (g.pr_state.count < sb) g.pr_state.allocate(sb);

    unsigned char *base = g.pr_state.get();
    PRArgs *d_args = reinterpret_cast<PRArgs *>(base);
    unsigned char *p = base + args_bytes;
    PRHeader *hdr = reinterpret_cast<PRHeader *>(p);
    p += sizeof(PRHeader);
    double *residual = reinterpret_cast<double *>(p);
    p += size_t(max_iter) * sizeof(double);
    double *dangling = reinterpret_cast<double *>(p);
    p += size_t(max_iter + 1) * sizeof(double);
    double *init_part = reinterpret_cast<double *>(p);
    p += size_t(init_chunks) * sizeof(double);
    uint32_t *init_count = reinterpret_cast<uint32_t *>(p);
    p += sizeof(uint32_t);
    uint32_t *blocks_done = reinterpret_cast<uint32_t *>(p);
    p += 4;
    const size_t zero_bytes = static_cast<size_t>(p - reinterpret_cast<unsigned char *>(hdr));
    p = base + args_bytes + up16(head);
    double2 *group_sum = reinterpret_cast<double2 *>(p);
    p += size_t(num_groups) * sizeof(double2);
    double2 *slots = reinterpret_cast<double2 *>(p);
    if (reinterpret_cast<uintptr_t>(base) % 256 || reinterpret_cast<uintptr_t>(group_sum) % 16 ||
        reinterpret_cast<uintptr_t>(slots) % 16 || reinterpret_cast<uintptr_t>(residual) % 8)
        fail(HYT_E_INTERNAL, "PageRank state layout is misaligned");

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
    for (int i = 0; i < 2; ++i) {
        a.rank[i] = g.rank[i].get();
        a.contrib[i] = g.contrib[i].get();
    }
    a.partial = reinterpret_cast<float2 *>(g.partial.get());
    a.ticket = g.ticket.get();
    a.hdr = hdr;
    a.residual = residual;
    a.dangling = dangling;
    a.num_tiles = g.num_tiles;
    a.num_chunks = static_cast<uint32_t>(g.num_chunks);
    a.V = static_cast<uint32_t>(V);
    a.damping = damping;
    a.base = personalized ? 0.0f : (1.0f - damping) / static_cast<float>(V);
    a.tolerance = tolerance;
    a.max_iter = max_iter;
    a.source = source;
    a.personalized = personalized ? 1u : 0u;
    a.use_cond = 0;
    a.red = PRSlots{slots, group_sum, blocks_done, static_cast<uint32_t>(num_slots),
                    static_cast<uint32_t>(num_groups)};
    a.tasks = g.pull_tasks.get();

    return PRSolveState{a, d_args, hdr, zero_bytes, init_part, init_count};
}

static void pr_check_header(const PRHeader &h) {
    if (h.error) fail(HYT_E_TIMEOUT, "PageRank: a bounded wait for a staged copy ran out");
    if (h.iter == 0) fail(HYT_E_INTERNAL, "PageRank made no progress");
}

// Grid of the per-iteration reduce kernel (fixed for a solve).
static unsigned pr_reduce_grid(const PRArgs &a) {
    return static_cast<unsigned>(std::max<uint32_t>(1u, std::min<uint32_t>(a.red.num_groups, 148u * 4)));
}

static void pr_init(const PRSolveState &st, uint64_t V, cudaStream_t s) {
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((V + kInitChunk - 1) / kInitChunk, 148ull * 8));
    pr_init_kernel<<<blocks, kInitThreads, 0, s>>>(st.d_args, st.init_part, st.init_count);
    HYT_CUDA(cudaGetLastError());
}

static void pr_solve(GraphImpl &g, bool personalized, uint32_t source, float damping, float tolerance,
                     uint32_t max_iter, uint32_t flags, cudaStream_t s, float *ranks_out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    const uint64_t V = g.V;
    PRSolveState st0 = pr_prepare(g, personalized, source, damping, tolerance, max_iter);
    PRArgs &a = st0.a;
    PRArgs *d_args = st0.d_args;
    PRHeader *hdr = st0.hdr;
    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    const int grid = pr_occupancy_grid();
    const bool staged = pr_use_staged(g);
    const int sgrid = pr_staged_grid();
    const void *kfunc = staged ? reinterpret_cast<const void *>(pr_staged_kernel)
                               : reinterpret_cast<const void *>(pr_iterate_kernel);
    const unsigned smem = static_cast<unsigned>(staged ? staged_shared_bytes(g.num_hot)
                                                       : pr_shared_bytes(g.num_hot, g.tile_cost));
    PRRange full{g.in_sources.get(), 0, g.num_chunks, 0, g.num_tiles, g.pull_tasks.get()};
    void *kargs[] = {&d_args, &full};
    const unsigned rgrid = pr_reduce_grid(a);
    auto launch = [&] {
        if (staged)
            pr_staged_kernel<<<sgrid, kStageThreads, smem, s>>>(d_args);
        else
            pr_iterate_kernel<<<grid, kPRThreads, smem, s>>>(d_args, full);
        pr_reduce_kernel<<<rgrid, kReduceThreads, 0, s>>>(d_args);
        HYT_CUDA(cudaGetLastError());
    };

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemsetAsync(hdr, 0, st0.zero_bytes, s));
    HYT_CUDA(cudaMemsetAsync(g.ticket.get(), 0, g.ticket.bytes(), s));

    uint32_t launches = 0, hot_launches = 0;
    double kernel_ms = 0.0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        HYT_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle cond;
        HYT_CUDA(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
        a.cond = cond;
        a.use_cond = 1;
    }
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(PRArgs), cudaMemcpyHostToDevice, s));
    pr_init(st0, V, s);
    ++launches;

    if (use_graph) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = a.cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        HYT_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaKernelNodeParams kp = {};
        kp.func = const_cast<void *>(kfunc);
        kp.gridDim = dim3(staged ? sgrid : grid);
        kp.blockDim = dim3(staged ? kStageThreads : kPRThreads);
        kp.sharedMemBytes = smem;
        kp.kernelParams = kargs;
        cudaGraphNode_t knode, rnode;
        HYT_CUDA(cudaGraphAddKernelNode(&knode, body, nullptr, 0, &kp));
        cudaKernelNodeParams rp = {};
        rp.func = reinterpret_cast<void *>(pr_reduce_kernel);
        rp.gridDim = dim3(rgrid);
        rp.blockDim = dim3(kReduceThreads);
        rp.kernelParams = kargs;
        HYT_CUDA(cudaGraphAddKernelNode(&rnode, body, &knode, 1, &rp));
        HYT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        HYT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        EventTimer kt;
        for (uint32_t i = 0; i < max_iter; ++i) {
            if (flags & HYT_RUN_PROFILE) kt.start(s);
            launch();
            launches += 2;
            if (flags & HYT_RUN_PROFILE) {
                kt.stop(s);
                const double ms = kt.ms();
                uint32_t done = 0;
                HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
                HYT_CUDA(cudaStreamSynchronize(s));
                kernel_ms += ms;
                ++hot_launches;
                if (done) break;
            } else if ((i & 3) == 3) {
                uint32_t done = 0;
                HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
                HYT_CUDA(cudaStreamSynchronize(s));
                if (done) break;
            }
        }
    }
    PRHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (use_graph) launches += 2 * h.iter;
    pr_check_header(h);
    if (ranks_out) graph_emit(g, ranks_out, g.rank[h.iter & 1].get(), s);

    if (stats) {
        stats->iterations = h.iter;
        stats->converged = h.converged;
        stats->residual = h.last_residual;
        stats->device_ms = total_ms;
        stats->kernel_ms = kernel_ms;
        stats->kernel_launches = hot_launches;
        stats->total_launches = launches;
        stats->edges_processed = uint64_t(h.iter) * g.E;
        stats->vertices_processed = uint64_t(h.iter) * V;
        // 4 B source id + 4 B gathered contribution per edge; 8 B CSC offset
        // + 4 B rank read + 4 B rank write + 4 B contribution write per vertex.
        stats->algorithmic_bytes = uint64_t(h.iter) * (8ull * g.E + 20ull * V);
    }
}

void pagerank_run(GraphImpl &g, const hyt_pagerank_params &p, float *ranks_out, hyt_run_stats *stats) {
    if (!(p.damping >= 0.0f && p.damping < 1.0f)) fail(HYT_E_INVALID, "PageRank damping_factor must be in [0, 1)");
    if (!(p.tolerance > 0.0f) || !std::isfinite(p.tolerance))
        fail(HYT_E_INVALID, "PageRank tolerance must be finite and positive");
    if (p.max_iterations == 0) fail(HYT_E_INVALID, "PageRank max_iterations must be greater than zero");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    pr_solve(g, false, 0, p.damping, p.tolerance, p.max_iterations, p.flags, s, ranks_out, stats);
}

void ppr_run(GraphImpl &g, const hyt_ppr_params &p, float *ranks_out, hyt_run_stats *stats) {
    if (!(p.restart > 0.0f && p.restart <= 1.0f)) fail(HYT_E_INVALID, "personalized PageRank restart must be in (0, 1]");
    if (!(p.tolerance > 0.0f) || !std::isfinite(p.tolerance))
        fail(HYT_E_INVALID, "personalized PageRank tolerance must be finite and positive");
    if (p.max_iterations == 0) fail(HYT_E_INVALID, "personalized PageRank max_iterations must be greater than zero");
    if (p.source >= g.V) fail(HYT_E_INVALID, "personalized PageRank source vertex is out of range");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    pr_solve(g, true, graph_vertex(g, p.source, s), 1.0f - p.restart, p.tolerance, p.max_iterations, p.flags, s,
             ranks_out, stats);
}

void pagerank_partitioned(GraphImpl &g, PullSource &src, bool personalized, uint32_t source, float damping,
                          float tolerance, uint32_t max_iter, cudaStream_t s, float *ranks_out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    PRSolveState st0 = pr_prepare(g, personalized, source, damping, tolerance, max_iter);
    const PRArgs &a = st0.a;
    const int grid = pr_occupancy_grid();
    const size_t smem = pr_shared_bytes(a.num_hot, a.tile_cost);

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemsetAsync(st0.hdr, 0, st0.zero_bytes, s));
    HYT_CUDA(cudaMemsetAsync(g.ticket.get(), 0, g.ticket.bytes(), s));
    HYT_CUDA(cudaMemcpyAsync(st0.d_args, &a, sizeof(PRArgs), cudaMemcpyHostToDevice, s));
    pr_init(st0, V, s);
    uint32_t launches = 1, hot = 0;
    PRHeader h{};
    for (uint32_t it = 0; it < max_iter; ++it) {
        src.begin_iteration(s);
        for (size_t p = 0; p < src.parts(); ++p) {
            const PullPart pp = src.part(p);
            if (pp.chunk_begin == pp.chunk_end && pp.tile_begin == pp.tile_end) continue;
            const uint32_t *base = src.acquire(p, s);
            const PRRange rg{base, pp.chunk_begin, pp.chunk_end, pp.tile_begin, pp.tile_end};
            pr_iterate_kernel<<<grid, kPRThreads, smem, s>>>(st0.d_args, rg);
            HYT_CUDA(cudaGetLastError());
            src.release(p, s);
            ++launches;
            ++hot;
        }
        pr_reduce_kernel<<<pr_reduce_grid(a), kReduceThreads, 0, s>>>(st0.d_args);
        HYT_CUDA(cudaGetLastError());
        ++launches;
        // the reduce kernel closed the iteration
        HYT_CUDA(cudaMemcpyAsync(&h, st0.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (h.error) break;
        if (h.iter != it + 1) fail(HYT_E_INTERNAL, "partitioned PageRank: an iteration left tasks unprocessed");
        if (h.done) break;
    }
    total.stop(s);
    const double total_ms = total.ms();
    pr_check_header(h);
    if (ranks_out) copy_from_device(ranks_out, g.rank[h.iter & 1].get(), V * sizeof(float), s);
    if (stats) {
        stats->iterations = h.iter;
        stats->converged = h.converged;
        stats->residual = h.last_residual;
        stats->device_ms = total_ms;
        stats->kernel_launches = hot;
        stats->total_launches = launches;
        stats->edges_processed = uint64_t(h.iter) * g.E;
        stats->vertices_processed = uint64_t(h.iter) * V;
        stats->algorithmic_bytes = uint64_t(h.iter) * (8ull * g.E + 20ull * V);
    }
}

}  // namespace hyt
