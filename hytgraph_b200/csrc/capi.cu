// extern "C" entry points of libhyt_core.so (declared in include/hyt/capi.h).
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <string>

#include "common.cuh"
#include "host_checks.hpp"
#include "scratch.cuh"
#include "graph.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string &msg) { g_last_error = msg; }
void clear_last_error() { g_last_error.clear(); }

cudaMemPool_t graph_pool(int device) {
    static std::mutex mu;
    static std::unordered_map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    HYT_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = kGraphPoolKeep;
    HYT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[device] = pool;
    return pool;
}

bool is_device_pointer(const void *p) {
    if (!p) return false;
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

PointerPlace pointer_place(const void *p, int current_device, int *pointer_device) {
    if (pointer_device) *pointer_device = -1;
    if (!p) return PointerPlace::kHost;
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return PointerPlace::kHost;
    }
    if (pointer_device) *pointer_device = attr.device;
    return classify_pointer(attr.type, attr.device, current_device);
}

void copy_to_device(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    const cudaMemcpyKind kind = is_device_pointer(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    HYT_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void copy_from_device(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (!bytes) return;
    const cudaMemcpyKind kind = is_device_pointer(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    HYT_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        HYT_CUDA(cudaGetDevice(&dev));
        HYT_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    }
    return n;
}

namespace {
void require_device() {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        fail(HYT_E_NO_DEVICE, "no CUDA device is available");
    }
}

GraphImpl &impl(hyt_graph *g) {
    if (!g) fail(HYT_E_INVALID, "graph handle is NULL");
    return g->impl;
}

void use_device(const GraphImpl &g) { HYT_CUDA(cudaSetDevice(g.device)); }

// HYT_LAUNCH=host selects host-driven launch loops instead of CUDA graphs
// with conditional nodes (same kernels, same work; profilers such as ncu
// cannot attribute kernels inside conditional graphs).
uint32_t launch_flags(uint32_t flags) {
    static const bool host = [] {
        const char *v = std::getenv("HYT_LAUNCH");
        return v && std::strcmp(v, "host") == 0;
    }();
    return host ? (flags | HYT_RUN_NO_GRAPH) : flags;
}
}  // namespace

}  // namespace hyt

using namespace hyt;

extern "C" {

const char *hyt_last_error(void) { return g_last_error.c_str(); }

int hyt_abi_version(void) { return HYT_ABI_VERSION; }

int hyt_device_count(int *count) {
    return guarded([&] {
        if (!count) fail(HYT_E_INVALID, "count is NULL");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

int hyt_copy(void *dst, const void *src, uint64_t bytes, void *stream) {
    return guarded([&] {
        if (!bytes) return;
        if (!dst || !src) fail(HYT_E_INVALID, "hyt_copy: NULL pointer");
        require_device();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        HYT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
        HYT_CUDA(cudaStreamSynchronize(s));
    });
}

int hyt_pinned_alloc(uint64_t bytes, void **out) {
    return guarded([&] {
        if (!out) fail(HYT_E_INVALID, "out is NULL");
        *out = nullptr;
        if (!bytes) fail(HYT_E_INVALID, "hyt_pinned_alloc: zero bytes");
        require_device();
        const cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            *out = nullptr;
            fail(HYT_E_OOM, std::string("cudaHostAlloc failed: ") + cudaGetErrorString(e));
        }
    });
}

int hyt_pinned_free(void *ptr) {
    return guarded([&] {
        if (ptr) HYT_CUDA(cudaFreeHost(ptr));
    });
}

int hyt_graph_create(const hyt_csr *csr, const hyt_graph_options *options, hyt_graph **out) {
    return guarded([&] {
        if (!csr || !out) fail(HYT_E_INVALID, "csr/out is NULL");
        *out = nullptr;
        require_device();
        hyt_graph_options opt = options_or_default(options);
        opt.device = resolve_device(opt.device);
        auto *g = new hyt_graph();
        try {
            g->impl.device = opt.device;
            HYT_CUDA(cudaSetDevice(opt.device));
            if (opt.stream) {
                g->impl.stream = static_cast<cudaStream_t>(opt.stream);
            } else {
                HYT_CUDA(cudaStreamCreateWithFlags(&g->impl.stream, cudaStreamNonBlocking));
                g->impl.own_stream = true;
            }
            g->impl.host_scratch.allocate(64);
            graph_create(g->impl, *csr, opt.flags);
        } catch (...) {
            if (g->impl.own_stream && g->impl.stream) cudaStreamDestroy(g->impl.stream);
            delete g;
            throw;
        }
        *out = g;
    });
}

int hyt_graph_destroy(hyt_graph *graph) {
    return guarded([&] {
        if (!graph) return;
        cudaSetDevice(graph->impl.device);
        cudaStreamSynchronize(graph->impl.stream);
        const bool own = graph->impl.own_stream;
        cudaStream_t s = graph->impl.stream;
        delete graph;
        if (own && s) cudaStreamDestroy(s);
    });
}

int hyt_graph_get_info(const hyt_graph *graph, hyt_graph_info *out) {
    return guarded([&] {
        if (!graph || !out) fail(HYT_E_INVALID, "graph/out is NULL");
        const GraphImpl &g = graph->impl;
        std::memset(out, 0, sizeof(*out));
        out->num_vertices = g.V;
        out->num_edges = g.E;
        out->weight_kind = g.weight_kind;
        out->flags = g.flags;
        out->device_bytes = g.device_bytes();
        out->pull_tiles = g.num_tiles;
        out->long_rows = g.num_long;
        out->max_in_degree = g.max_in_degree;
        out->max_out_degree = g.max_out_degree;
        out->dangling_vertices = g.dangling;
        out->build_ms = g.build_ms;
        out->device = g.device;
    });
}

int hyt_graph_copy_csc(const hyt_graph *graph, uint64_t *in_offsets, uint32_t *in_sources) {
    return guarded([&] {
        if (!graph || !in_offsets || !in_sources) fail(HYT_E_INVALID, "NULL argument");
        const GraphImpl &g = graph->impl;
        HYT_CUDA(cudaSetDevice(g.device));
        graph_copy_csc(g, in_offsets, in_sources);
    });
}

int hyt_pagerank(hyt_graph *graph, const hyt_pagerank_params *params, float *ranks_out, hyt_run_stats *stats) {
    return guarded([&] {
        if (!params) fail(HYT_E_INVALID, "params is NULL");
        GraphImpl &g = impl(graph);
        use_device(g);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        hyt_pagerank_params p = *params;
        p.flags = launch_flags(p.flags);
        pagerank_run(g, p, ranks_out, stats);
    });
}

int hyt_ppr_multi(hyt_graph *graph, const uint32_t *sources, uint32_t num_sources, float restart, float tolerance,
                  uint32_t max_iterations, float *ranks_out, hyt_run_stats *stats) {
    return guarded([&] {
        GraphImpl &g = impl(graph);
        use_device(g);
        ppr_multi(g, sources, num_sources, restart, tolerance, max_iterations, ranks_out, stats);
    });
}

int hyt_ppr(hyt_graph *graph, const hyt_ppr_params *params, float *ranks_out, hyt_run_stats *stats) {
    return guarded([&] {
        if (!params) fail(HYT_E_INVALID, "params is NULL");
        GraphImpl &g = impl(graph);
        use_device(g);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        hyt_ppr_params p = *params;
        p.flags = launch_flags(p.flags);
        ppr_run(g, p, ranks_out, stats);
    });
}

int hyt_sssp(hyt_graph *graph, const hyt_sssp_params *params, uint32_t *dist_out, hyt_run_stats *stats) {
    return guarded([&] {
        if (!params) fail(HYT_E_INVALID, "params is NULL");
        GraphImpl &g = impl(graph);
        use_device(g);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        hyt_sssp_params p = *params;
        p.flags = launch_flags(p.flags);
        sssp_run(g, p, dist_out, stats);
    });
}

int hyt_sssp_multi(hyt_graph *graph, const uint32_t *sources, uint32_t num_sources, uint32_t max_rounds,
                   uint32_t *dist_out, hyt_run_stats *stats) {
    return guarded([&] {
        GraphImpl &g = impl(graph);
        use_device(g);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        sssp_multi(g, sources, num_sources, max_rounds, launch_flags(0), g.stream, dist_out, stats);
    });
}

int hyt_sssp_noalloc(const hyt_csr *csr, uint32_t source, uint32_t *dist_out, void *stream, hyt_run_stats *stats) {
    return guarded([&] {
        if (!csr || !dist_out) fail(HYT_E_INVALID, "csr/dist_out is NULL");
        require_device();
        sssp_noalloc(*csr, source, dist_out, stream, stats);
    });
}

int hyt_rmat_generate(const hyt_rmat_params *params, int on_device, hyt_csr_buffers *out) {
    return guarded([&] {
        if (!params) fail(HYT_E_INVALID, "params is NULL");
        if (on_device) require_device();
        rmat_generate(*params, on_device != 0, out);
    });
}

int hyt_csr_buffers_free(hyt_csr_buffers *b) {
    return guarded([&] {
        if (!b) return;
        if (b->on_device) {
            if (b->row_offsets) cudaFree(b->row_offsets);
            if (b->column_indices) cudaFree(b->column_indices);
            if (b->weights) cudaFree(b->weights);
        } else {
            std::free(b->row_offsets);
            std::free(b->column_indices);
            std::free(b->weights);
        }
        std::memset(b, 0, sizeof(*b));
    });
}

int hyt_hub_sort(const hyt_csr *csr, double hub_fraction, uint32_t *vertex_order, double *scores,
                 uint64_t *hub_count, hyt_reorder_stats *stats) {
    return guarded([&] {
        if (!csr) fail(HYT_E_INVALID, "csr is NULL");
        require_device();
        hub_sort(*csr, hub_fraction, vertex_order, scores, hub_count, stats);
    });
}

int hyt_csr_reorder(const hyt_csr *csr, const uint32_t *vertex_order, int on_device, hyt_csr_buffers *out,
                    hyt_reorder_stats *stats) {
    return guarded([&] {
        if (!csr) fail(HYT_E_INVALID, "csr is NULL");
        require_device();
        csr_reorder(*csr, vertex_order, on_device != 0, out, stats);
    });
}

int hyt_load_edge_list(const char *path, uint64_t num_vertices, int weighted, int on_device,
                       hyt_csr_buffers *out, hyt_load_stats *stats) {
    return guarded([&] {
        require_device();
        load_edge_list(path, num_vertices, weighted != 0, on_device != 0, out, stats);
    });
}

int hyt_csr_from_edges(const uint32_t *src, const uint32_t *dst, const void *weights, uint32_t weight_kind,
                       uint64_t num_edges, uint64_t num_vertices, int on_device, hyt_csr_buffers *out,
                       hyt_load_stats *stats) {
    return guarded([&] {
        require_device();
        csr_from_edges(src, dst, weights, weight_kind, num_edges, num_vertices, on_device != 0, out, stats);
    });
}

int hyt_csr_save(const char *path, const hyt_csr *csr) {
    return guarded([&] {
        if (!csr) fail(HYT_E_INVALID, "csr is NULL");
        require_device();
        csr_save(path, *csr);
    });
}

int hyt_csr_load(const char *path, int on_device, hyt_csr_buffers *out, hyt_load_stats *stats) {
    return guarded([&] {
        require_device();
        csr_load(path, on_device != 0, out, stats);
    });
}

int hyt_pagerank_contributions(hyt_graph *graph, const float *current_ranks, float damping,
                               double *contributions) {
    return guarded([&] {
        if (!graph) fail(HYT_E_INVALID, "graph is NULL");
        pagerank_contributions(graph->impl, current_ranks, damping, contributions, nullptr);
    });
}

int hyt_sssp_contributions(const float *current_distances, const float *candidate_distances, uint64_t n,
                           float tolerance, double *contributions) {
    return guarded([&] {
        require_device();
        sssp_contributions(current_distances, candidate_distances, n, tolerance, contributions);
    });
}

int hyt_contribution_schedule(const uint64_t *item_indices, const double *contributions, uint64_t n,
                              int deterministic_tie_break, double zero_contribution_epsilon,
                              uint64_t *ordered_items, hyt_contribution_metrics *metrics) {
    return guarded([&] {
        require_device();
        contribution_schedule(item_indices, contributions, n, deterministic_tie_break != 0, zero_contribution_epsilon,
                              ordered_items, metrics);
    });
}

int hyt_partition_contributions(const double *vertex_contributions, uint64_t num_vertices, const uint64_t *bounds,
                                uint64_t num_partitions, double *out) {
    return guarded([&] {
        require_device();
        partition_contributions(vertex_contributions, num_vertices, bounds, num_partitions, out);
    });
}

int hyt_trim_device_memory(int device) {
    return guarded([&] {
        require_device();
        int cur = 0;
        HYT_CUDA(cudaGetDevice(&cur));
        HYT_CUDA(cudaSetDevice(device));
        HYT_CUDA(cudaDeviceSynchronize());
        HYT_CUDA(cudaMemPoolTrimTo(graph_pool(device), 0));
        HYT_CUDA(cudaMemPoolTrimTo(scratch_pool(), 0));
        HYT_CUDA(cudaSetDevice(cur));
    });
}

int hyt_pick_sources(const uint64_t *row_offsets, uint64_t num_vertices, uint64_t seed, uint32_t count,
                     uint32_t *out) {
    return guarded([&] { pick_sources(row_offsets, num_vertices, seed, count, out); });
}

}  // extern "C"
