// Seeded R-MAT generator (Chakrabarti, Zhan, Faloutsos 2004) and seeded
// source selection.
//
// Edge draw i (0 <= i < edge_factor * 2^scale) descends `scale` levels of the
// adjacency matrix; level l picks quadrant (0,0) / (0,1) / (1,0) / (1,1) with
// probabilities a / b / c / d = 1-a-b-c from a 32-bit uniform.  Uniforms come
// from a counter-based splitmix64 stream (word j of draw i is
// splitmix64(seed + golden * (16 i + j))), so every draw is independent of
// evaluation order: the host generator (threads) and the device generator
// (one thread per draw) emit identical edges.  Self-loops and duplicate
// (u, v) pairs are dropped; edges are sorted by (source, destination).
// Weights are a hash of (u, v) and the seed, uniform in [weight_min,
// weight_max], hence independent of edge order too.
//
// The reference ships no generator (its datasets/ folder is empty); this one
// feeds the same bytes to the GPU path and to the CPU oracle.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "common.cuh"
#include "prims.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kNoEdge = ~0ull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct RmatKey {
    uint64_t seed;
    uint32_t scale;
    uint32_t ta, tab, tabc;  // cumulative thresholds scaled to 2^32
};

__host__ __device__ __forceinline__ uint64_t rmat_draw(const RmatKey &k, uint64_t i) {
    uint32_t src = 0, dst = 0;
    uint64_t word = 0;
    for (uint32_t l = 0; l < k.scale; ++l) {
        if ((l & 1u) == 0) word = mix64(k.seed + kGolden * (16ull * i + (l >> 1)));
        const uint32_t r = (l & 1u) ? static_cast<uint32_t>(word >> 32) : static_cast<uint32_t>(word);
        const uint32_t bit = 1u << (k.scale - 1 - l);
        if (r < k.ta) {
        } else if (r < k.tab) {
            dst |= bit;
        } else if (r < k.tabc) {
            src |= bit;
        } else {
            src |= bit;
            dst |= bit;
        }
    }
    if (src == dst) return kNoEdge;
    return (uint64_t(src) << 32) | dst;
}

__host__ __device__ __forceinline__ uint32_t rmat_weight(uint64_t wseed, uint64_t key, uint32_t wmin, uint32_t span) {
    return wmin + static_cast<uint32_t>(mix64(key ^ wseed) % span);
}

RmatKey make_key(const hyt_rmat_params &p) {
    if (p.scale < 1 || p.scale > 31) fail(HYT_E_INVALID, "R-MAT scale must be in [1, 31]");
    if (p.edge_factor == 0) fail(HYT_E_INVALID, "R-MAT edge_factor must be positive");
    const double d = 1.0 - p.a - p.b - p.c;
    if (!(p.a >= 0 && p.b >= 0 && p.c >= 0 && d >= -1e-12))
        fail(HYT_E_INVALID, "R-MAT probabilities must be non-negative and sum to at most 1");
    if (p.weight_max < p.weight_min) fail(HYT_E_INVALID, "R-MAT weight_max < weight_min");
    auto thr = [](double x) -> uint32_t {
        const double v = x * 4294967296.0;
        return v >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<uint32_t>(v);
    };
    RmatKey k;
    k.seed = p.seed;
    k.scale = p.scale;
    k.ta = thr(p.a);
    k.tab = thr(p.a + p.b);
    k.tabc = thr(p.a + p.b + p.c);
    return k;
}

uint64_t weight_seed(uint64_t seed) { return mix64(seed ^ 0x5EEDF00DCAFEBABEull); }

// ------------------------------- device --------------------------------
__global__ void rmat_draw_kernel(RmatKey k, uint64_t n, uint64_t *keys) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) keys[i] = rmat_draw(k, i);
}

__global__ void unique_flags_kernel(const uint64_t *keys, uint64_t n, uint8_t *flags) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride)
        flags[i] = keys[i] != kNoEdge && (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void csr_from_keys_kernel(const uint64_t *keys, uint64_t E, uint64_t V, uint64_t wseed, uint32_t wmin,
                                     uint32_t span, uint64_t *off, uint32_t *cols, uint32_t *w) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e <= E; e += stride) {
        const int64_t prev = (e == 0) ? -1 : static_cast<int64_t>(keys[e - 1] >> 32);
        const int64_t cur = (e == E) ? static_cast<int64_t>(V) : static_cast<int64_t>(keys[e] >> 32);
        for (int64_t v = prev + 1; v <= cur; ++v) off[v] = e;
        if (e < E) {
            const uint64_t key = keys[e];
            cols[e] = static_cast<uint32_t>(key);
            if (w) w[e] = rmat_weight(wseed, key, wmin, span);
        }
    }
}

void generate_device(const hyt_rmat_params &p, const RmatKey &k, hyt_csr_buffers *out) {
    cudaStream_t s = nullptr;
    HYT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    const uint64_t V = 1ull << p.scale;
    const uint64_t n = uint64_t(p.edge_factor) * V;
    DeviceArray<uint64_t> keys(n);
    rmat_draw_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(k, n, keys.get());
    HYT_CUDA(cudaGetLastError());
    // sentinel kNoEdge has every bit set and sorts last
    prims::sort_keys_u64(keys.get(), n, 64, s);
    uint64_t E = 0;
    {
        DeviceArray<uint8_t> flags(n);
        unique_flags_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(keys.get(), n, flags.get());
        HYT_CUDA(cudaGetLastError());
        DeviceArray<uint64_t> uniq(n);
        E = prims::select_flagged_u64(keys.get(), flags.get(), uniq.get(), n, s);
        keys = std::move(uniq);
    }
    const bool weighted = !(p.weight_min == 0 && p.weight_max == 0);
    uint64_t *off = nullptr;
    uint32_t *cols = nullptr, *w = nullptr;
    HYT_CUDA(cudaMalloc(&off, (V + 1) * sizeof(uint64_t)));
    HYT_CUDA(cudaMalloc(&cols, std::max<uint64_t>(E, 1) * sizeof(uint32_t) + 16));
    if (weighted) HYT_CUDA(cudaMalloc(&w, std::max<uint64_t>(E, 1) * sizeof(uint32_t) + 16));
    const uint32_t span = p.weight_max - p.weight_min + 1u;
    csr_from_keys_kernel<<<grid_for(E + 1, 256, 148 * 16), 256, 0, s>>>(keys.get(), E, V, weight_seed(p.seed),
                                                                         p.weight_min, span ? span : 1u, off, cols, w);
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaStreamSynchronize(s));
    out->num_vertices = V;
    out->num_edges = E;
    out->row_offsets = off;
    out->column_indices = cols;
    out->weights = w;
    out->on_device = 1;
    out->weight_kind = w ? HYT_WEIGHTS_U32 : HYT_WEIGHTS_NONE;
}

// -------------------------------- host ---------------------------------
template <class F>
void parallel_for(uint64_t n, F &&f) {
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    if (n < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    const uint64_t step = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const uint64_t b = t * step, e = std::min<uint64_t>(n, b + step);
        if (b >= e) break;
        th.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto &x : th) x.join();
}

void generate_host(const hyt_rmat_params &p, const RmatKey &k, hyt_csr_buffers *out) {
    const uint64_t V = 1ull << p.scale;
    const uint64_t n = uint64_t(p.edge_factor) * V;
    std::vector<uint64_t> keys(n);
    parallel_for(n, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) keys[i] = rmat_draw(k, i);
    });
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    while (!keys.empty() && keys.back() == kNoEdge) keys.pop_back();
    const uint64_t E = keys.size();
    const bool weighted = !(p.weight_min == 0 && p.weight_max == 0);
    auto *off = static_cast<uint64_t *>(std::malloc((V + 1) * sizeof(uint64_t)));
    auto *cols = static_cast<uint32_t *>(std::malloc(std::max<uint64_t>(E, 1) * sizeof(uint32_t)));
    uint32_t *w = weighted ? static_cast<uint32_t *>(std::malloc(std::max<uint64_t>(E, 1) * sizeof(uint32_t))) : nullptr;
    if (!off || !cols || (weighted && !w)) {
        std::free(off);
        std::free(cols);
        std::free(w);
        fail(HYT_E_OOM, "host allocation for the R-MAT graph failed");
    }
    const uint64_t wseed = weight_seed(p.seed);
    const uint32_t span = p.weight_max - p.weight_min + 1u;
    uint64_t e = 0;
    for (uint64_t v = 0; v < V; ++v) {
        off[v] = e;
        while (e < E && (keys[e] >> 32) == v) {
            cols[e] = static_cast<uint32_t>(keys[e]);
            if (w) w[e] = rmat_weight(wseed, keys[e], p.weight_min, span ? span : 1u);
            ++e;
        }
    }
    off[V] = E;
    out->num_vertices = V;
    out->num_edges = E;
    out->row_offsets = off;
    out->column_indices = cols;
    out->weights = w;
    out->on_device = 0;
    out->weight_kind = w ? HYT_WEIGHTS_U32 : HYT_WEIGHTS_NONE;
}

}  // namespace

void rmat_generate(const hyt_rmat_params &p, bool on_device, hyt_csr_buffers *out) {
    if (!out) fail(HYT_E_INVALID, "output buffers pointer is NULL");
    std::memset(out, 0, sizeof(*out));
    const RmatKey k = make_key(p);
    if (on_device)
        generate_device(p, k, out);
    else
        generate_host(p, k, out);
}

void pick_sources(const uint64_t *row_offsets, uint64_t V, uint64_t seed, uint32_t count, uint32_t *out) {
    if (!row_offsets || (!out && count)) fail(HYT_E_INVALID, "NULL pointer");
    if (V == 0) fail(HYT_E_INVALID, "graph has no vertices");
    uint64_t with_edges = 0;
    for (uint64_t v = 0; v < V; ++v) with_edges += row_offsets[v + 1] > row_offsets[v];
    if (with_edges == 0 && count) fail(HYT_E_INVALID, "graph has no vertex with out-degree > 0");
    const uint64_t want_unique = std::min<uint64_t>(count, with_edges);
    std::vector<uint32_t> chosen;
    uint64_t j = 0;
    while (chosen.size() < count) {
        const uint64_t v = mix64(seed + kGolden * (++j)) % V;
        if (row_offsets[v + 1] == row_offsets[v]) continue;
        if (chosen.size() < want_unique &&
            std::find(chosen.begin(), chosen.end(), static_cast<uint32_t>(v)) != chosen.end())
            continue;
        chosen.push_back(static_cast<uint32_t>(v));
    }
    std::copy(chosen.begin(), chosen.end(), out);
}

}  // namespace hyt
