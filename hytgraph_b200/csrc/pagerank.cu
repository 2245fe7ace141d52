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
#include "pagerank_core.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

using namespace prc;

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

    const PRBuffers b = buffers(a, it);
    const PRState ps = make_state(a, a.dangling[it]);
    const uint64_t pol = dev::policy_evict_last();
    const uint64_t n_chunks = rg.chunk_end - rg.chunk_begin;
    const uint64_t total_tasks = n_chunks + (rg.tile_end - rg.tile_begin);
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
        for (int k = 0; k < 8; ++k) hc[k] = b.ccur[hv[k]];
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
            chunk_task<true>(a, ps, b, rg.in_src, s_hot, rg.chunk_begin + task, pol, lane, res, dang);
        } else {
            tile_task<true>(a, ps, b, rg.in_src, s_hot, sv, rg.tile_begin + (task - n_chunks), pol, lane, res, dang);
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
