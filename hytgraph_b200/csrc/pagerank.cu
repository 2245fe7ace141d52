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
// One persistent kernel per iteration.  CTAs pull tasks from a counter:
//   chunk tasks  -- 8192-edge slices of rows with in-degree >= 4096; each
//                   CTA writes a compensated partial, the last arriving CTA
//                   of a row merges the partials in chunk order;
//   tile tasks   -- merge-path tiles of consecutive rows; the tile's
//                   in-sources are read with 128-bit streaming loads, the
//                   contributions gathered into shared memory, then reduced
//                   thread-per-row (in-degree < 32) or warp-per-row.
// Results are deterministic: every sum has a fixed association order.
// The last CTA to finish an iteration evaluates the stop rule and, inside a
// CUDA graph, ends the conditional while-loop.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "graph.cuh"
#include "hybrid.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

constexpr uint32_t kWarpRowDegree = 16;  // rows with more in-edges are summed by a whole warp

struct PRHeader {
    uint32_t iter;       // iterations completed
    uint32_t done;
    uint32_t converged;
    uint32_t pad;
    double last_residual;
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
    uint32_t *task_counter;  // [max_iter]
    uint32_t *finished;      // [max_iter]
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
};

struct PRState {
    // per-iteration scalars
    float damping, base, teleport_scale;
    float dshare;  // PR: d * dangling / n
    float tele;    // PPR: (1-d) + d * dangling
    uint32_t source;
    bool personalized;
};

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
constexpr int kBatch = 16;

template <class Sink>
__device__ __forceinline__ void gather_span(const uint32_t *in_src, const float *ccur, const float *s_hot, uint64_t lo,
                                            uint64_t hi, uint64_t pol, int lane, Sink &&sink) {
    const uint32_t n = static_cast<uint32_t>(hi - lo);
    const uint32_t *src = in_src + lo;
    for (uint32_t base = 0; base < n; base += 32 * kBatch) {
        uint32_t id[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t i = base + 32 * k + lane;
            id[k] = (i < n) ? dev::ld_stream(src + i) : 0u;
        }
        float v[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            v[k] = 0.0f;
            if (!(id[k] & kHotTag)) v[k] = dev::ld_keep(ccur + id[k], pol);
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k)
            if (id[k] & kHotTag) v[k] = s_hot[id[k] & ~kHotTag];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t i = base + 32 * k + lane;
            if (i < n) sink(i, v[k]);
        }
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

// One launch processes chunk tasks [chunk_begin, chunk_end) and tiles
// [tile_begin, tile_end); in_src is the base of the source ids, addressed by
// global edge index (a device array, a staging slot offset by its first
// edge, or mapped host memory).  partial = 1: the iteration is closed later
// by pr_iteration_end_kernel.
struct PRRange {
    const uint32_t *in_src;
    uint64_t chunk_begin, chunk_end, tile_begin, tile_end;
    uint32_t partial;
};

__global__ void __launch_bounds__(kPRThreads, 1) pr_iterate_kernel(const PRArgs *__restrict__ args, PRRange rg) {
    extern __shared__ __align__(16) float s_dyn[];
    __shared__ double s_red[32];

    const PRArgs a = *args;
    const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
    if (*(volatile uint32_t *)&a.hdr->done) return;

    const float *cur = (it & 1) ? a.rank[1] : a.rank[0];
    float *nxt = (it & 1) ? a.rank[0] : a.rank[1];
    const float *ccur = (it & 1) ? a.contrib[1] : a.contrib[0];
    float *cnxt = (it & 1) ? a.contrib[0] : a.contrib[1];

    PRState ps;
    ps.damping = a.damping;
    ps.source = a.source;
    ps.personalized = a.personalized != 0;
    const double dmass = a.dangling[it];
    ps.dshare = __fadd_rn(a.base, static_cast<float>(static_cast<double>(a.damping) * dmass / static_cast<double>(a.V)));
    ps.tele = static_cast<float>((1.0 - static_cast<double>(a.damping)) + static_cast<double>(a.damping) * dmass);

    const uint64_t pol = dev::policy_evict_last();
    const uint64_t n_chunks = rg.chunk_end - rg.chunk_begin;
    const uint64_t total_tasks = n_chunks + (rg.tile_end - rg.tile_begin);
    const uint32_t *in_src = rg.in_src;
    double res = 0.0, dang = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Hot-source contributions for this iteration, loaded once per CTA.
    float *s_hot = s_dyn;
    for (uint32_t i0 = 0; i0 < a.num_hot; i0 += 8 * kPRThreads) {
        uint32_t hv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * kPRThreads + threadIdx.x;
            hv[k] = (i < a.num_hot) ? a.hot_vertex[i] : 0u;
        }
        float hc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) hc[k] = ccur[hv[k]];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = i0 + k * kPRThreads + threadIdx.x;
            if (i < a.num_hot) s_hot[i] = hc[k];
        }
    }
    __syncthreads();
    float *sv = s_dyn + a.num_hot + warp * (2 * a.tile_cost + 8);
    const uint64_t nwarps = uint64_t(gridDim.x) * (kPRThreads / 32);

    // Static round-robin over tasks: every task costs at most one chunk of
    // edges, so warps receive balanced work without a shared counter.
    for (uint64_t task = uint64_t(blockIdx.x) * (kPRThreads / 32) + warp; task < total_tasks; task += nwarps) {
        if (task < n_chunks) {
            // ---- slice of a long row -------------------------------------
            const uint2 t = a.chunk_tasks[rg.chunk_begin + task];
            const LongRow L = a.long_rows[t.x];
            const uint64_t rb = a.in_off[L.row], re = a.in_off[L.row + 1];
            const uint64_t b = rb + uint64_t(t.y) * kLongChunk;
            const uint64_t e = (b + kLongChunk < re) ? b + kLongChunk : re;
            dev::CSum acc;
            gather_span(in_src, ccur, s_hot, b, e, pol, lane, [&](uint32_t, float v) { acc.add(v); });
            acc = dev::warp_reduce(acc);
            uint32_t last = 0;
            if (lane == 0) {
                a.partial[L.first_chunk + t.y] = make_float2(acc.s, acc.c);
                __threadfence();
                const uint32_t tk = atomicAdd(&a.ticket[t.x], 1u) + 1u;
                last = (tk % L.num_chunks == 0) ? 1u : 0u;
            }
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                // the last arriving warp merges every chunk of the row, in a
                // fixed order: lane j takes chunks j, j+32, ...
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
                if (lane == 0) finalize_row(a, ps, L.row, row.value(), cur, nxt, cnxt, res, dang);
            }
        } else {
            // ---- merge-path tile of consecutive rows ---------------------
            const uint64_t k = rg.tile_begin + (task - n_chunks);
            const uint32_t r0 = a.tile_start[k];
            const uint32_t r1 = a.tile_start[k + 1];
            if (r0 == r1) continue;
            const uint64_t last_b = a.in_off[r1 - 1], last_e = a.in_off[r1];
            const uint32_t rl = (last_e - last_b >= a.tile_cost) ? r1 - 1 : r1;  // long last row is chunked
            const uint64_t e0 = a.in_off[r0];
            const uint64_t e1 = (rl == r1) ? last_e : last_b;
            const uint64_t a0 = e0;
            gather_span(in_src, ccur, s_hot, e0, e1, pol, lane, [&](uint32_t i, float v) { sv[i] = v; });
            __syncwarp();
            for (uint32_t rb = r0; rb < rl; rb += 32) {
                const uint32_t r = rb + lane;
                const bool active = r < rl;
                const uint64_t b = active ? a.in_off[r] : 0;
                const uint64_t e = active ? a.in_off[r + 1] : 0;
                if (active && e - b < kWarpRowDegree) {
                    dev::CSum acc;
                    for (uint64_t x = b; x < e; ++x) acc.add(sv[x - a0]);
                    finalize_row(a, ps, r, acc.value(), cur, nxt, cnxt, res, dang);
                }
                uint32_t big = __ballot_sync(0xffffffffu, active && (e - b >= kWarpRowDegree));
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint64_t bb = __shfl_sync(0xffffffffu, b, src);
                    const uint64_t ee = __shfl_sync(0xffffffffu, e, src);
                    dev::CSum acc;
                    for (uint64_t x = bb + lane; x < ee; x += 32) acc.add(sv[x - a0]);
                    acc = dev::warp_reduce(acc);
                    if (lane == 0) finalize_row(a, ps, rb + src, acc.value(), cur, nxt, cnxt, res, dang);
                }
            }
            __syncwarp();
        }
    }

    const double bres = dev::block_sum(res, s_red);
    __syncthreads();
    const double bdang = dev::block_sum(dang, s_red);
    if (threadIdx.x == 0) {
        atomicAdd(&a.residual[it], bres);
        atomicAdd(&a.dangling[it + 1], bdang);
        if (!rg.partial) {
            __threadfence();
            const uint32_t t = atomicAdd(&a.finished[it], 1u);
            if (t == gridDim.x - 1) {
                __threadfence();
                end_iteration(a, it);
            }
        }
    }
}

// Closes an iteration whose tasks ran as several partial launches.
__global__ void pr_iteration_end_kernel(const PRArgs *__restrict__ args) {
    const PRArgs a = *args;
    if (a.hdr->done) return;
    end_iteration(a, a.hdr->iter);
}

__global__ void pr_init_kernel(const PRArgs *__restrict__ args) {
    __shared__ double s_red[32];
    const PRArgs a = *args;
    const uint32_t V = a.V;
    const float r0_uniform = __fdiv_rn(1.0f, static_cast<float>(V));
    double dang = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const float r0 = a.personalized ? (v == a.source ? 1.0f : 0.0f) : r0_uniform;
        a.rank[0][v] = r0;
        const uint32_t od = a.out_deg[v];
        a.contrib[0][v] = od ? __fdiv_rn(r0, static_cast<float>(od)) : 0.0f;
        if (od == 0) dang += r0;
    }
    const double b = dev::block_sum(dang, s_red);
    if (threadIdx.x == 0 && b != 0.0) atomicAdd(&a.dangling[0], b);
}

size_t state_bytes(uint32_t max_iter) {
    return sizeof(PRHeader) + size_t(max_iter) * (2 * sizeof(uint32_t) + sizeof(double)) +
           size_t(max_iter + 1) * sizeof(double) + 64;
}

int pr_occupancy_grid() {
    static int grid = 0;
    if (grid == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaFuncSetAttribute(pr_iterate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPRSmemMax)));
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_iterate_kernel, kPRThreads, kPRSmemMax));
        grid = sm_count() * std::max(per_sm, 1);
    }
    return grid;
}

struct SolveOut {
    uint32_t iterations;
    uint32_t converged;
    double residual;
};

}  // namespace

// Shared by PageRank and personalized PageRank.
// Workspaces, device state layout and kernel arguments of one solve.
struct PRSolveState {
    PRArgs a;
    PRArgs *d_args;
    PRHeader *hdr;
    size_t zero_bytes;
};

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
    const size_t sb = state_bytes(max_iter) + sizeof(PRArgs) + 256;
    if (g.pr_state.count < sb) g.pr_state.allocate(sb);

    unsigned char *base = g.pr_state.get();
    PRArgs *d_args = reinterpret_cast<PRArgs *>(base);
    unsigned char *p = base + ((sizeof(PRArgs) + 255) & ~size_t(255));
    PRHeader *hdr = reinterpret_cast<PRHeader *>(p);
    p += sizeof(PRHeader);
    double *residual = reinterpret_cast<double *>(p);
    p += size_t(max_iter) * sizeof(double);
    double *dangling = reinterpret_cast<double *>(p);
    p += size_t(max_iter + 1) * sizeof(double);
    uint32_t *task_counter = reinterpret_cast<uint32_t *>(p);
    p += size_t(max_iter) * sizeof(uint32_t);
    uint32_t *finished = reinterpret_cast<uint32_t *>(p);
    p += size_t(max_iter) * sizeof(uint32_t);
    const size_t zero_bytes = static_cast<size_t>(p - reinterpret_cast<unsigned char *>(hdr));

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
    a.task_counter = task_counter;
    a.finished = finished;
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

    return PRSolveState{a, d_args, hdr, zero_bytes};
}

static void pr_solve(GraphImpl &g, bool personalized, uint32_t source, float damping, float tolerance,
                     uint32_t max_iter, uint32_t flags, cudaStream_t s, float *ranks_out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    const uint64_t V = g.V;
    PRSolveState st0 = pr_prepare(g, personalized, source, damping, tolerance, max_iter);
    PRArgs &a = st0.a;
    PRArgs *d_args = st0.d_args;
    PRHeader *hdr = st0.hdr;
    const size_t zero_bytes = st0.zero_bytes;
    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    const int grid = pr_occupancy_grid();

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemsetAsync(hdr, 0, zero_bytes, s));
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
    pr_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    ++launches;
    PRRange full{g.in_sources.get(), 0, g.num_chunks, 0, g.num_tiles, 0};

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
        void *kargs[] = {&d_args, &full};
        kp.func = reinterpret_cast<void *>(pr_iterate_kernel);
        kp.gridDim = dim3(grid);
        kp.blockDim = dim3(kPRThreads);
        kp.sharedMemBytes = static_cast<unsigned>(pr_shared_bytes(g.num_hot, g.tile_cost));
        kp.kernelParams = kargs;
        cudaGraphNode_t knode;
        HYT_CUDA(cudaGraphAddKernelNode(&knode, body, nullptr, 0, &kp));
        HYT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        HYT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        EventTimer kt;
        for (uint32_t i = 0; i < max_iter; ++i) {
            if (flags & HYT_RUN_PROFILE) kt.start(s);
            pr_iterate_kernel<<<grid, kPRThreads, pr_shared_bytes(g.num_hot, g.tile_cost), s>>>(d_args, full);
            HYT_CUDA(cudaGetLastError());
            ++launches;
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
    if (use_graph) launches += h.iter;
    if (h.iter == 0) fail(HYT_E_INTERNAL, "PageRank made no progress");
    if (ranks_out) copy_from_device(ranks_out, g.rank[h.iter & 1].get(), V * sizeof(float), s);

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
    pr_solve(g, true, p.source, 1.0f - p.restart, p.tolerance, p.max_iterations, p.flags, s, ranks_out, stats);
}

void pagerank_partitioned(GraphImpl &g, PullSource &src, bool personalized, uint32_t source, float damping,
                          float tolerance, uint32_t max_iter, cudaStream_t s, float *ranks_out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    PRSolveState st0 = pr_prepare(g, personalized, source, damping, tolerance, max_iter);
    const PRArgs &a = st0.a;
    const int grid = pr_occupancy_grid();
    const size_t smem = pr_shared_bytes(a.num_hot, a.tile_cost);

    EventTimer total, kt;
    total.start(s);
    HYT_CUDA(cudaMemsetAsync(st0.hdr, 0, st0.zero_bytes, s));
    HYT_CUDA(cudaMemsetAsync(g.ticket.get(), 0, g.ticket.bytes(), s));
    HYT_CUDA(cudaMemcpyAsync(st0.d_args, &a, sizeof(PRArgs), cudaMemcpyHostToDevice, s));
    pr_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(st0.d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 1, hot = 0;
    PRHeader h{};
    for (uint32_t it = 0; it < max_iter; ++it) {
        src.begin_iteration(s);
        for (size_t p = 0; p < src.parts(); ++p) {
            const PullPart pp = src.part(p);
            if (pp.chunk_begin == pp.chunk_end && pp.tile_begin == pp.tile_end) continue;
            const uint32_t *base = src.acquire(p, s);
            const PRRange rg{base, pp.chunk_begin, pp.chunk_end, pp.tile_begin, pp.tile_end, 1u};
            pr_iterate_kernel<<<grid, kPRThreads, smem, s>>>(st0.d_args, rg);
            HYT_CUDA(cudaGetLastError());
            src.release(p, s);
            ++launches;
            ++hot;
        }
        pr_iteration_end_kernel<<<1, 1, 0, s>>>(st0.d_args);
        HYT_CUDA(cudaGetLastError());
        ++launches;
        HYT_CUDA(cudaMemcpyAsync(&h, st0.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
    }
    total.stop(s);
    const double total_ms = total.ms();
    if (h.iter == 0) fail(HYT_E_INTERNAL, "PageRank made no progress");
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
