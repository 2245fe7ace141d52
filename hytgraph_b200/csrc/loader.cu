// Graph construction and loading: hyt_load_edge_list, hyt_csr_from_edges,
// hyt_csr_save, hyt_csr_load.
//
// Text edge lists follow GraphLoader::load_edge_list
// (src/graph/graph_loader.cpp:39-179).  The file's bytes stream into HBM
// through the pinned ring; the GPU finds the line starts (a select over
// byte positions), parses every line in its own thread with the
// reference's record rules (the extraction rules of `stream >> uint64_t`,
// `stream >> float` and `stream >> std::string`, as libstdc++ applies them),
// and reports the first failing line in file order with the reference's
// message.  A weight whose strtof value is one correctly rounded float
// division (at most 7 significant and 10 fractional digits, no exponent)
// is converted on the GPU; the host re-parses the rare other forms with
// the exact rules.  The kept records are compacted in file order and the
// GPU builds the CSR: a stable radix sort of (source, destination[,
// weight]) pairs on the source bits keeps the file order within a source
// and keeps parallel edges (the reference's std::stable_sort by source),
// row offsets come from a lower-bound search per vertex, and the sorted
// pairs are unpacked into the column and weight arrays.
//
// The binary CSR format is this library's own (the reference reads text
// only); its layout and checksum are declared in hyt/capi.h.  Loading to
// the device streams the payload through a ring of pinned buffers, each
// filled by its own reader thread and copied on its own stream, then checks
// the checksum and the CSR structure on the GPU.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"
#include "scratch.cuh"

namespace hyt {
namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

unsigned grid_sm(unsigned per_sm) { return static_cast<unsigned>(sm_count()) * per_sm; }

unsigned host_threads(uint64_t work_bytes, uint64_t bytes_per_thread = uint64_t(4) << 20) {
    unsigned n = std::thread::hardware_concurrency();
    if (n == 0) n = 1;
    n = std::min(n, 64u);
    const uint64_t by_work = std::max<uint64_t>(1, work_bytes / bytes_per_thread);
    return static_cast<unsigned>(std::min<uint64_t>(n, by_work));
}

// Runs f(i) for i in [0, n) on n threads (f(0) on the caller); the first
// exception thrown by any of them is rethrown.
template <class F>
void parallel_for(unsigned n, F &&f) {
    std::vector<std::exception_ptr> errs(n);
    std::vector<std::thread> th;
    th.reserve(n ? n - 1 : 0);
    for (unsigned i = 1; i < n; ++i)
        th.emplace_back([&, i] {
            try {
                f(i);
            } catch (...) {
                errs[i] = std::current_exception();
            }
        });
    try {
        if (n) f(0);
    } catch (...) {
        errs[0] = std::current_exception();
    }
    for (auto &t : th) t.join();
    for (auto &e : errs)
        if (e) std::rethrow_exception(e);
}

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) ::close(fd);
    }
};

// ------------------------------ text records ------------------------------

enum : int { kRecOk = 0, kRecMalformed = 2, kRecRange = 3, kRecMissingWeight = 4, kRecTrailing = 5 };

__host__ __device__ inline bool ws_char(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
__host__ __device__ inline bool trim_char(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

__host__ __device__ inline const char *skip_ws(const char *p, const char *e) {
    while (p < e && ws_char(*p)) ++p;
    return p;
}

// `stream >> uint64_t`: whitespace, an optional sign, decimal digits; no
// digit or overflow fails; '-' negates modulo 2^64.
__host__ __device__ bool extract_u64(const char *&p, const char *e, uint64_t &out) {
    p = skip_ws(p, e);
    bool neg = false, overflow = false;
    int digits = 0;
    uint64_t v = 0;
    if (p < e && (*p == '-' || *p == '+')) {
        neg = *p == '-';
        ++p;
    }
    while (p < e && *p >= '0' && *p <= '9') {
        const uint64_t d = static_cast<uint64_t>(*p - '0');
        if (v > (~uint64_t(0) - d) / 10) overflow = true;
        v = v * 10 + d;
        ++digits;
        ++p;
    }
    if (!digits || overflow) return false;
    out = neg ? uint64_t(0) - v : v;
    return true;
}

// `stream >> float`: the characters num_get accumulates ([sign], leading
// zeros collapsed, digits with one '.', then 'e' with an optional sign
// once a digit was seen), converted by strtof; nothing converted,
// unconverted accumulated characters or an infinite value fail.
bool extract_f32(const char *&p, const char *e, float &out) {
    p = skip_ws(p, e);
    char small[96];
    std::string big;
    size_t n = 0;
    auto put = [&](char c) {
        if (n + 1 < sizeof(small)) {
            small[n++] = c;
        } else {
            if (big.empty()) big.assign(small, n);
            big.push_back(c);
            ++n;
        }
    };
    bool mant = false, dec = false, sci = false;
    if (p < e && (*p == '+' || *p == '-')) put(*p++);
    while (p < e && *p == '0') {
        if (!mant) {
            put('0');
            mant = true;
        }
        ++p;
    }
    while (p < e) {
        const char c = *p;
        if (c == '.' && !dec && !sci) {
            put('.');
            dec = true;
        } else if (c >= '0' && c <= '9') {
            put(c);
            mant = true;
        } else if ((c == 'e' || c == 'E') && !sci && mant) {
            put('e');
            sci = true;
            ++p;
            if (p >= e) break;
            if (*p == '+' || *p == '-') {
                put(*p);
            } else {
                continue;
            }
        } else {
            break;
        }
        ++p;
    }
    const char *tok = big.empty() ? (small[n] = '\0', small) : big.c_str();
    char *end = nullptr;
    const float v = std::strtof(tok, &end);
    if (end == tok || *end != '\0' || std::isinf(v)) return false;
    out = v;
    return true;
}

// The record of one line, on the host (the exact rules, for lines the GPU
// hands back): status kRecOk (edge), 1 (blank / comment) or an error kind.
int host_record(const char *a, const char *z, uint64_t V, bool weighted, uint32_t &s32, uint32_t &d32, uint32_t &w32) {
    while (a < z && trim_char(*a)) ++a;
    while (z > a && trim_char(z[-1])) --z;
    if (a == z || *a == '#') return 1;
    uint64_t s = 0, d = 0;
    float wt = 0.0f;
    const char *q = a;
    if (!extract_u64(q, z, s) || !extract_u64(q, z, d)) return kRecMalformed;
    if (s >= V || d >= V) return kRecRange;
    if (weighted && !extract_f32(q, z, wt)) return kRecMissingWeight;
    if (skip_ws(q, z) != z) return kRecTrailing;
    s32 = static_cast<uint32_t>(s);
    d32 = static_cast<uint32_t>(d);
    std::memcpy(&w32, &wt, 4);
    return kRecOk;
}

// ------------------------------ records on the GPU ------------------------

constexpr uint8_t kLineSkip = 1;  // blank or comment
constexpr uint8_t kLineSlow = 6;  // a weight the GPU leaves to the host

__global__ void count_newlines_kernel(const char *__restrict__ text, uint64_t n, unsigned long long *count) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint64_t c = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) c += text[i] == '\n';
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

struct LineStart {
    const char *text;
    __device__ bool operator()(uint64_t p) const { return p == 0 || text[p - 1] == '\n'; }
};

// `stream >> float` for the forms whose strtof result one correctly rounded
// float division gives: [sign] digits [. digits], at most 7 significant
// digits and 10 fractional digits, no exponent.  m and 10^k are then exact
// floats and m / 10^k rounds once, as strtof does.  Returns 1 (value), 0
// (no number: the reference fails) or 2 (another form: the host decides).
__device__ int extract_f32_fast(const char *&p, const char *e, float &out) {
    p = skip_ws(p, e);
    bool neg = false, dec = false, mant = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    uint32_t m = 0;
    int sig = 0, frac = 0;
    for (; p < e; ++p) {
        const char c = *p;
        if (c == '.' && !dec) {
            dec = true;
        } else if (c >= '0' && c <= '9') {
            mant = true;
            if (dec) ++frac;
            if (m == 0 && c == '0') continue;  // leading zero
            if (++sig > 7) return 2;
            m = m * 10 + static_cast<uint32_t>(c - '0');
        } else {
            break;
        }
    }
    if (!mant) return 0;
    if (p < e && (*p == 'e' || *p == 'E')) return 2;
    if (frac > 10) return 2;
    const float pow10[11] = {1e0f, 1e1f, 1e2f, 1e3f, 1e4f, 1e5f, 1e6f, 1e7f, 1e8f, 1e9f, 1e10f};
    const float v = __fdiv_rn(static_cast<float>(m), pow10[frac]);
    out = neg ? -v : v;
    return 1;
}

// One thread per line: the line's status and, for an edge, its fields.
__global__ void parse_lines_kernel(const char *__restrict__ text, uint64_t size, const uint64_t *__restrict__ ls,
                                   uint64_t L, uint64_t V, bool weighted, uint8_t *__restrict__ status,
                                   uint32_t *__restrict__ s_out, uint32_t *__restrict__ d_out,
                                   uint32_t *__restrict__ w_out, unsigned long long *__restrict__ first_error,
                                   unsigned long long *__restrict__ slow) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < L; i += stride) {
        const char *a = text + ls[i];
        const char *z = text + (i + 1 < L ? ls[i + 1] : size);
        while (a < z && trim_char(*a)) ++a;
        while (z > a && trim_char(z[-1])) --z;
        uint8_t st = kRecOk;
        uint32_t s32 = 0, d32 = 0, w32 = 0;
        if (a == z || *a == '#') {
            st = kLineSkip;
        } else {
            uint64_t sv = 0, dv = 0;
            const char *q = a;
            if (!extract_u64(q, z, sv) || !extract_u64(q, z, dv)) {
                st = kRecMalformed;
            } else if (sv >= V || dv >= V) {
                st = kRecRange;
            } else {
                float wt = 0.0f;
                const int r = weighted ? extract_f32_fast(q, z, wt) : 1;
                if (r == 0) {
                    st = kRecMissingWeight;
                } else if (r == 2) {
                    st = kLineSlow;
                } else if (skip_ws(q, z) != z) {
                    st = kRecTrailing;
                }
                s32 = static_cast<uint32_t>(sv);
                d32 = static_cast<uint32_t>(dv);
                w32 = __float_as_uint(wt);
            }
        }
        status[i] = st;
        s_out[i] = s32;
        d_out[i] = d32;
        if (w_out) w_out[i] = w32;
        if (st >= kRecMalformed && st <= kRecTrailing) atomicMin(first_error, static_cast<unsigned long long>(i));
        if (st == kLineSlow) atomicAdd(slow, 1ull);
    }
}

// The host's verdicts for the lines the GPU left to it.
__global__ void patch_lines_kernel(const uint64_t *__restrict__ idx, const uint8_t *__restrict__ st,
                                   const uint32_t *__restrict__ sv, const uint32_t *__restrict__ dv,
                                   const uint32_t *__restrict__ wv, uint64_t n, uint8_t *__restrict__ status,
                                   uint32_t *__restrict__ s, uint32_t *__restrict__ d, uint32_t *__restrict__ w) {
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = idx[k];
        status[i] = st[k];
        s[i] = sv[k];
        d[i] = dv[k];
        if (w) w[i] = wv[k];
    }
}

__global__ void line_bounds_kernel(const uint64_t *__restrict__ ls, uint64_t L, uint64_t size,
                                   const uint64_t *__restrict__ idx, uint64_t n, uint64_t *__restrict__ b,
                                   uint64_t *__restrict__ e) {
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = idx[k];
        b[k] = ls[i];
        e[k] = i + 1 < L ? ls[i + 1] : size;
    }
}

__global__ void edge_flags_kernel(const uint8_t *__restrict__ status, uint64_t L, uint64_t *__restrict__ flag) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < L; i += uint64_t(gridDim.x) * blockDim.x)
        flag[i] = status[i] == kRecOk;
}

__global__ void compact_edges_kernel(const uint8_t *__restrict__ status, const uint64_t *__restrict__ pos, uint64_t L,
                                     const uint32_t *__restrict__ s, const uint32_t *__restrict__ d,
                                     const uint32_t *__restrict__ w, uint32_t *__restrict__ cs,
                                     uint32_t *__restrict__ cd, uint32_t *__restrict__ cw) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < L; i += uint64_t(gridDim.x) * blockDim.x) {
        if (status[i] != kRecOk) continue;
        const uint64_t k = pos[i];
        cs[k] = s[i];
        cd[k] = d[i];
        if (w) cw[k] = w[i];
    }
}

__global__ void slow_flags_kernel(const uint8_t *__restrict__ status, uint64_t L, uint8_t *__restrict__ flag) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < L; i += uint64_t(gridDim.x) * blockDim.x)
        flag[i] = status[i] == kLineSlow;
}

// ------------------------------ CSR construction --------------------------

__global__ void first_bad_edge_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t E,
                                      uint64_t V, unsigned long long *first) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < E; i += stride)
        if (src[i] >= V || dst[i] >= V) atomicMin(first, static_cast<unsigned long long>(i));
}

// *unsorted = 1 when some source is smaller than the one before it.
__global__ void descending_pair_kernel(const uint32_t *__restrict__ src, uint64_t E, uint32_t *unsorted) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    bool bad = false;
    for (uint64_t i = 1 + blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < E; i += stride)
        bad |= src[i] < src[i - 1];
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(unsorted, 1u);
}

// Sort keys (sources) and values (destination, with the weight's bits in
// the high half when weighted).
__global__ void pack_edges_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                                  const uint32_t *__restrict__ w, uint64_t E, uint32_t *__restrict__ keys,
                                  uint64_t *__restrict__ vals64, uint32_t *__restrict__ vals32) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < E; i += stride) {
        keys[i] = src[i];
        if (w) {
            vals64[i] = (uint64_t(w[i]) << 32) | dst[i];
        } else {
            vals32[i] = dst[i];
        }
    }
}

// off[v] = number of sorted keys below v, for v in [0, V].
__global__ void offsets_from_sorted_kernel(const uint32_t *__restrict__ keys, uint64_t E, uint64_t V,
                                           uint64_t *__restrict__ off) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v <= V; v += stride) {
        uint64_t lo = 0, hi = E;  // first index with keys[i] >= v
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < v) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        off[v] = lo;
    }
}

__global__ void unpack_edges_kernel(const uint64_t *__restrict__ vals64, uint64_t E, uint32_t *__restrict__ cols,
                                    uint32_t *__restrict__ w) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < E; i += stride) {
        const uint64_t x = vals64[i];
        cols[i] = static_cast<uint32_t>(x);
        w[i] = static_cast<uint32_t>(x >> 32);
    }
}

// Output buffers of a call: cudaMalloc'd (device) or malloc'd (host), freed
// again if the call fails before handing them over.
struct Output {
    hyt_csr_buffers *o;
    bool armed = true;
    Output(hyt_csr_buffers *out, uint64_t V, uint64_t E, uint32_t wkind, bool on_device) : o(out) {
        std::memset(o, 0, sizeof(*o));
        o->num_vertices = V;
        o->num_edges = E;
        o->on_device = on_device ? 1u : 0u;
        o->weight_kind = wkind;
        o->row_offsets = static_cast<uint64_t *>(alloc((V + 1) * 8));
        o->column_indices = static_cast<uint32_t *>(alloc(E * 4));
        if (wkind != HYT_WEIGHTS_NONE) o->weights = static_cast<uint32_t *>(alloc(E * 4));
    }
    void *alloc(size_t bytes) {
        void *p = nullptr;
        if (o->on_device) {
            HYT_CUDA(cudaMalloc(&p, bytes ? bytes : 16));
        } else {
            p = std::malloc(bytes ? bytes : 16);
            if (!p) fail(HYT_E_OOM, "host allocation failed");
        }
        return p;
    }
    ~Output() {
        if (armed) hyt_csr_buffers_free(o);
    }
};

int key_bits(uint64_t V) {
    if (V <= 1) return 1;
    return 64 - __builtin_clzll(V - 1);
}

// Builds the CSR of device edge arrays into `out` (device or host).
// Returns the construction's device time.
double build_csr(const uint32_t *src, const uint32_t *dst, const uint32_t *w, uint64_t E, uint64_t V, uint32_t wkind,
                 bool on_device, hyt_csr_buffers *out, cudaStream_t s) {
    const bool weighted = wkind != HYT_WEIGHTS_NONE;
    Output res(out, V, E, weighted ? wkind : HYT_WEIGHTS_NONE, on_device);
    std::unique_ptr<Scratch<uint64_t>> off_s;
    std::unique_ptr<Scratch<uint32_t>> cols_s, w_s;
    uint64_t *off = out->row_offsets;
    uint32_t *cols = out->column_indices, *wo = out->weights;
    if (!on_device) {
        off_s = std::make_unique<Scratch<uint64_t>>(V + 1, s);
        cols_s = std::make_unique<Scratch<uint32_t>>(E, s);
        off = off_s->get();
        cols = cols_s->get();
        if (weighted) {
            w_s = std::make_unique<Scratch<uint32_t>>(E, s);
            wo = w_s->get();
        }
    }
    EventTimer t;
    if (E) {
        // sources already in order (a file in CSR order): the stable sort
        // is the identity, so the edges are copied as they are
        Scratch<uint32_t> unsorted(1, s);
        HYT_CUDA(cudaMemsetAsync(unsorted.get(), 0, 4, s));
        descending_pair_kernel<<<grid_sm(8), 256, 0, s>>>(src, E, unsorted.get());
        HYT_CUDA(cudaGetLastError());
        uint32_t h_unsorted = 0;
        HYT_CUDA(cudaMemcpyAsync(&h_unsorted, unsorted.get(), 4, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (!h_unsorted) {
            t.start(s);
            HYT_CUDA(cudaMemcpyAsync(cols, dst, E * 4, cudaMemcpyDeviceToDevice, s));
            if (weighted) HYT_CUDA(cudaMemcpyAsync(wo, w, E * 4, cudaMemcpyDeviceToDevice, s));
            offsets_from_sorted_kernel<<<grid_for(V + 1, 256), 256, 0, s>>>(src, E, V, off);
            HYT_CUDA(cudaGetLastError());
            t.stop(s);
        } else {
            // every buffer first, so the timed region holds only device work
            Scratch<uint32_t> k0(E, s), k1(E, s);
            std::unique_ptr<Scratch<uint64_t>> v64a, v64b;
            std::unique_ptr<Scratch<uint32_t>> v32b;
            if (weighted) {
                v64a = std::make_unique<Scratch<uint64_t>>(E, s);
                v64b = std::make_unique<Scratch<uint64_t>>(E, s);
            } else {
                v32b = std::make_unique<Scratch<uint32_t>>(E, s);
            }
            // unweighted: the destinations are sorted straight into the output
            uint32_t *v32a = weighted ? nullptr : cols;
            const int bits = key_bits(V);
            cub::DoubleBuffer<uint32_t> kb(k0.get(), k1.get());
            cub::DoubleBuffer<uint64_t> vb64(weighted ? v64a->get() : nullptr, weighted ? v64b->get() : nullptr);
            cub::DoubleBuffer<uint32_t> vb32(v32a, weighted ? nullptr : v32b->get());
            size_t tb = 0;
            if (weighted) {
                HYT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb64, static_cast<int64_t>(E), 0, bits, s));
            } else {
                HYT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb32, static_cast<int64_t>(E), 0, bits, s));
            }
            Scratch<uint8_t> tmp(tb, s);
            HYT_CUDA(cudaStreamSynchronize(s));
            t.start(s);
            pack_edges_kernel<<<grid_for(E, 256), 256, 0, s>>>(src, dst, weighted ? w : nullptr, E, k0.get(),
                                                              weighted ? v64a->get() : nullptr, v32a);
            HYT_CUDA(cudaGetLastError());
            if (weighted) {
                HYT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, kb, vb64, static_cast<int64_t>(E), 0, bits, s));
                unpack_edges_kernel<<<grid_for(E, 256), 256, 0, s>>>(vb64.Current(), E, cols, wo);
                HYT_CUDA(cudaGetLastError());
            } else {
                HYT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, kb, vb32, static_cast<int64_t>(E), 0, bits, s));
                if (vb32.Current() != cols)
                    HYT_CUDA(cudaMemcpyAsync(cols, vb32.Current(), E * 4, cudaMemcpyDeviceToDevice, s));
            }
            offsets_from_sorted_kernel<<<grid_for(V + 1, 256), 256, 0, s>>>(kb.Current(), E, V, off);
            HYT_CUDA(cudaGetLastError());
            t.stop(s);
            HYT_CUDA(cudaStreamSynchronize(s));  // the scratch above is released on this stream
        }
    } else {
        t.start(s);
        HYT_CUDA(cudaMemsetAsync(off, 0, (V + 1) * 8, s));
        t.stop(s);
    }
    if (!on_device) {
        HYT_CUDA(cudaMemcpyAsync(out->row_offsets, off, (V + 1) * 8, cudaMemcpyDeviceToHost, s));
        if (E) HYT_CUDA(cudaMemcpyAsync(out->column_indices, cols, E * 4, cudaMemcpyDeviceToHost, s));
        if (weighted && E) HYT_CUDA(cudaMemcpyAsync(out->weights, wo, E * 4, cudaMemcpyDeviceToHost, s));
    }
    HYT_CUDA(cudaStreamSynchronize(s));
    res.armed = false;
    return t.ms();
}

uint64_t construction_bytes(uint64_t E, uint64_t V, bool weighted) {
    // edges read (source, destination[, weight]) and written (destination
    // [, weight]); offsets written
    return E * (weighted ? 20 : 12) + 8 * (V + 1);
}

// ------------------------------ binary format -----------------------------

struct FileHeader {
    char magic[8];
    uint32_t version;
    uint32_t weight_kind;
    uint64_t num_vertices;
    uint64_t num_edges;
    uint64_t payload_bytes;
    uint64_t checksum;
    uint64_t header_check;
    uint64_t reserved;
};
static_assert(sizeof(FileHeader) == 64, "header is 64 bytes");

constexpr char kMagic[8] = {'H', 'Y', 'T', 'C', 'S', 'R', '0', '1'};
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t pad8(uint64_t b) { return (b + 7) & ~uint64_t(7); }

uint64_t header_check(const FileHeader &h) {
    uint64_t words[6];
    std::memcpy(words, &h, sizeof(words));
    uint64_t c = 0;
    for (uint64_t x : words) c = splitmix64(c ^ x);
    return c;
}

struct Layout {
    uint64_t off_bytes, cols_bytes, w_bytes, payload;
    uint64_t cols_at, w_at;  // payload offsets
    Layout(uint64_t V, uint64_t E, bool weighted) {
        off_bytes = 8 * (V + 1);
        cols_bytes = 4 * E;
        w_bytes = weighted ? 4 * E : 0;
        cols_at = off_bytes;
        w_at = cols_at + pad8(cols_bytes);
        payload = w_at + pad8(w_bytes);
    }
};

// Checksum terms of a section seen as 32-bit values (little-endian pairs
// form the 64-bit words), word index starting at word_base.
__global__ void checksum_kernel(const uint32_t *__restrict__ a, uint64_t n32, uint64_t word_base,
                                unsigned long long *__restrict__ sum) {
    const uint64_t words = (n32 + 1) / 2;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint64_t acc = 0;
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < words; j += stride) {
        const uint64_t lo = a[2 * j];
        const uint64_t hi = 2 * j + 1 < n32 ? a[2 * j + 1] : 0;
        acc += splitmix64((lo | (hi << 32)) ^ ((word_base + j) * kGolden));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(sum, static_cast<unsigned long long>(acc));
}

uint64_t host_checksum(const uint32_t *a, uint64_t n32, uint64_t word_base) {
    const uint64_t words = (n32 + 1) / 2;
    const unsigned T = host_threads(words * 8, uint64_t(16) << 20);
    std::vector<uint64_t> part(T, 0);
    parallel_for(T, [&](unsigned t) {
        const uint64_t b = words * t / T, e = words * (t + 1) / T;
        uint64_t acc = 0;
        for (uint64_t j = b; j < e; ++j) {
            const uint64_t lo = a[2 * j];
            const uint64_t hi = 2 * j + 1 < n32 ? a[2 * j + 1] : 0;
            acc += splitmix64((lo | (hi << 32)) ^ ((word_base + j) * kGolden));
        }
        part[t] = acc;
    });
    uint64_t s = 0;
    for (uint64_t x : part) s += x;
    return s;
}

enum : uint32_t { kBadOffsets = 1u, kBadTerminal = 2u, kBadColumn = 4u };

__global__ void check_structure_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ cols, uint64_t V,
                                       uint64_t E, uint32_t *bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t b = 0;
    for (uint64_t v = tid; v < V; v += stride)
        if (off[v + 1] < off[v]) b |= kBadOffsets;
    for (uint64_t e = tid; e < E; e += stride)
        if (cols[e] >= V) b |= kBadColumn;
    if (tid == 0) {
        if (off[0] != 0) b |= kBadOffsets;
        if (off[V] != E) b |= kBadTerminal;
    }
    if (b) atomicOr(bad, b);
}

uint32_t host_structure(const uint64_t *off, const uint32_t *cols, uint64_t V, uint64_t E) {
    const unsigned T = host_threads(std::max(V, E) * 4, uint64_t(16) << 20);
    std::vector<uint32_t> part(T, 0);
    parallel_for(T, [&](unsigned t) {
        uint32_t b = 0;
        for (uint64_t v = V * t / T, e = V * (t + 1) / T; v < e; ++v)
            if (off[v + 1] < off[v]) b |= kBadOffsets;
        for (uint64_t i = E * t / T, e = E * (t + 1) / T; i < e; ++i)
            if (cols[i] >= V) b |= kBadColumn;
        part[t] = b;
    });
    uint32_t b = 0;
    for (uint32_t x : part) b |= x;
    if (off[0] != 0) b |= kBadOffsets;
    if (off[V] != E) b |= kBadTerminal;
    return b;
}

void fail_structure(uint32_t b) {
    if (b & kBadOffsets) fail(HYT_E_INVALID, "row offsets must start at 0 and be non-decreasing");
    if (b & kBadTerminal) fail(HYT_E_INVALID, "terminal row offset must equal the number of edges");
    if (b & kBadColumn) fail(HYT_E_INVALID, "column index contains an invalid destination vertex ID");
}

void write_all(int fd, const void *p, uint64_t n, const std::string &path) {
    const char *c = static_cast<const char *>(p);
    while (n) {
        const ssize_t k = ::write(fd, c, std::min<uint64_t>(n, uint64_t(1) << 30));
        if (k < 0) {
            if (errno == EINTR) continue;
            fail(HYT_E_IO, "error while writing file: " + path);
        }
        c += k;
        n -= static_cast<uint64_t>(k);
    }
}

// Reads n bytes at `at`; `what` names the file in the error message.
void read_all(int fd, void *p, uint64_t n, uint64_t at, const std::string &what) {
    char *c = static_cast<char *>(p);
    while (n) {
        const ssize_t k = ::pread(fd, c, std::min<uint64_t>(n, uint64_t(1) << 30), static_cast<off_t>(at));
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0) fail(HYT_E_IO, what);
        c += k;
        n -= static_cast<uint64_t>(k);
        at += static_cast<uint64_t>(k);
    }
}

// Pinned staging ring for device loads, allocated on first use and kept.
constexpr int kRing = 8;
constexpr uint64_t kRingBytes = uint64_t(32) << 20;
struct PinnedRing {
    std::mutex mu;
    void *buf[kRing] = {};
    bool ready = false;
    void init() {
        if (ready) return;
        for (int i = 0; i < kRing; ++i) HYT_CUDA(cudaHostAlloc(&buf[i], kRingBytes, cudaHostAllocPortable));
        ready = true;
    }
};
PinnedRing &ring() {
    static PinnedRing r;
    return r;
}

// One contiguous piece of the payload bound for one device array.
struct Piece {
    uint64_t file_at;
    char *dst;
    uint64_t bytes;
};

// Streams file pieces into device memory through the pinned ring: reader
// thread t owns ring buffer t and its own stream, reads its pieces (t,
// t + threads, ...) and copies each one once the buffer's previous copy has
// finished.  Returns the number of reader threads.
unsigned stream_to_device(int fd, const std::vector<Piece> &pieces, const std::string &path) {
    int dev = 0;
    HYT_CUDA(cudaGetDevice(&dev));
    PinnedRing &r = ring();
    std::lock_guard<std::mutex> lk(r.mu);
    r.init();
    const unsigned threads = static_cast<unsigned>(std::min<size_t>(kRing, std::max<size_t>(pieces.size(), 1)));
    parallel_for(threads, [&](unsigned t) {
        HYT_CUDA(cudaSetDevice(dev));
        cudaStream_t cs = nullptr;
        cudaEvent_t done = nullptr;
        HYT_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        HYT_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        struct Release {
            cudaStream_t s;
            cudaEvent_t e;
            ~Release() {
                cudaStreamSynchronize(s);
                cudaEventDestroy(e);
                cudaStreamDestroy(s);
            }
        } rel{cs, done};
        bool pending = false;
        for (size_t k = t; k < pieces.size(); k += threads) {
            if (pending) HYT_CUDA(cudaEventSynchronize(done));  // this buffer's last copy
            read_all(fd, r.buf[t], pieces[k].bytes, pieces[k].file_at, path);
            HYT_CUDA(cudaMemcpyAsync(pieces[k].dst, r.buf[t], pieces[k].bytes, cudaMemcpyHostToDevice, cs));
            HYT_CUDA(cudaEventRecord(done, cs));
            pending = true;
        }
    });
    return threads;
}

std::vector<Piece> cut(uint64_t file_at, char *dst, uint64_t bytes) {
    std::vector<Piece> v;
    for (uint64_t d = 0; d < bytes; d += kRingBytes) v.push_back({file_at + d, dst + d, std::min(kRingBytes, bytes - d)});
    return v;
}

}  // namespace

// ------------------------------ entry points ------------------------------

void csr_from_edges(const uint32_t *src, const uint32_t *dst, const void *weights, uint32_t wkind, uint64_t E,
                    uint64_t V, bool on_device, hyt_csr_buffers *out, hyt_load_stats *stats) {
    const auto t0 = Clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!out) fail(HYT_E_INVALID, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    if (V > (uint64_t(1) << 32)) fail(HYT_E_INVALID, "num_vertices must be at most 2^32 (32-bit vertex ids)");
    if (wkind != HYT_WEIGHTS_NONE && wkind != HYT_WEIGHTS_U32 && wkind != HYT_WEIGHTS_F32)
        fail(HYT_E_INVALID, "unknown weight kind");
    if (E && (!src || !dst)) fail(HYT_E_INVALID, "edge arrays are NULL");
    if (E && wkind != HYT_WEIGHTS_NONE && !weights) fail(HYT_E_INVALID, "weights are NULL");
    if (E && V == 0) fail(HYT_E_INVALID, "edges need at least one vertex");
    StreamHold st;
    cudaStream_t s = st.s;
    EventTimer whole;
    whole.start(s);
    std::unique_ptr<Scratch<uint32_t>> sh, dh, wh;
    const uint32_t *ds = device_view(src, E, sh, s);
    const uint32_t *dd = device_view(dst, E, dh, s);
    const uint32_t *dw = wkind != HYT_WEIGHTS_NONE ? device_view(static_cast<const uint32_t *>(weights), E, wh, s)
                                                   : nullptr;
    if (E) {
        Scratch<unsigned long long> first(1, s);
        HYT_CUDA(cudaMemsetAsync(first.get(), 0xFF, 8, s));
        first_bad_edge_kernel<<<grid_for(E, 256), 256, 0, s>>>(ds, dd, E, V, first.get());
        HYT_CUDA(cudaGetLastError());
        unsigned long long h = 0;
        HYT_CUDA(cudaMemcpyAsync(&h, first.get(), 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (h != ~0ull) fail(HYT_E_INVALID, "edge " + std::to_string(h) + " has a vertex ID >= num_vertices");
    }
    const double kms = build_csr(ds, dd, dw, E, V, wkind, on_device, out, s);
    whole.stop(s);
    if (stats) {
        stats->device_ms = whole.ms();
        stats->kernel_ms = kms;
        stats->num_edges = E;
        stats->kernel_bytes = construction_bytes(E, V, wkind != HYT_WEIGHTS_NONE);
        stats->threads = 1;
        stats->total_ms = ms_since(t0);
    }
}

void load_edge_list(const char *path, uint64_t V, bool weighted, bool on_device, hyt_csr_buffers *out,
                    hyt_load_stats *stats) {
    const auto t0 = Clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!out || !path) fail(HYT_E_INVALID, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    if (V > (uint64_t(1) << 32)) fail(HYT_E_INVALID, "num_vertices must be at most 2^32 (32-bit vertex ids)");
    const std::string p(path);
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) fail(HYT_E_IO, "GraphLoader::load_edge_list: unable to open file: " + p);
    struct stat sb {};
    if (::fstat(f.fd, &sb) != 0) fail(HYT_E_IO, "GraphLoader::load_edge_list: error while reading file: " + p);
    const uint64_t size = static_cast<uint64_t>(sb.st_size);
    StreamHold st;
    cudaStream_t s = st.s;
    // 1. the raw bytes into HBM (zero padding after them)
    Scratch<char> text(size + 64, s);
    HYT_CUDA(cudaMemsetAsync(text.get() + size, 0, 64, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    const unsigned threads = size ? stream_to_device(f.fd, cut(0, text.get(), size),
                                                        "GraphLoader::load_edge_list: error while reading file: " + p) : 1;
    const double read_ms = ms_since(t0);
    EventTimer whole;
    whole.start(s);
    // 2. line starts: position 0 and every position after a '\n'
    uint64_t L = 0;
    if (size) {
        Scratch<unsigned long long> cnt(1, s);
        HYT_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, s));
        count_newlines_kernel<<<grid_sm(8), 256, 0, s>>>(text.get(), size - 1, cnt.get());
        unsigned long long h = 0;
        HYT_CUDA(cudaMemcpyAsync(&h, cnt.get(), 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        L = h + 1;  // newlines before the last byte each start a line
    }
    Scratch<uint64_t> ls(L + 1, s), nsel(1, s);
    if (L) {
        thrust::counting_iterator<uint64_t> it(0);
        LineStart pred{text.get()};
        size_t tb = 0;
        HYT_CUDA(cub::DeviceSelect::If(nullptr, tb, it, ls.get(), nsel.get(), static_cast<int64_t>(size), pred, s));
        Scratch<uint8_t> tmp(tb, s);
        HYT_CUDA(cub::DeviceSelect::If(tmp.get(), tb, it, ls.get(), nsel.get(), static_cast<int64_t>(size), pred, s));
    }
    // 3. every line's record
    Scratch<uint8_t> status(L, s);
    Scratch<uint32_t> sv(L, s), dv(L, s);
    std::unique_ptr<Scratch<uint32_t>> wv;
    if (weighted) wv = std::make_unique<Scratch<uint32_t>>(L, s);
    Scratch<unsigned long long> first(1, s), slow(1, s);
    HYT_CUDA(cudaMemsetAsync(first.get(), 0xFF, 8, s));
    HYT_CUDA(cudaMemsetAsync(slow.get(), 0, 8, s));
    if (L)
        parse_lines_kernel<<<grid_sm(8), 256, 0, s>>>(text.get(), size, ls.get(), L, V, weighted, status.get(), sv.get(),
                                                      dv.get(), weighted ? wv->get() : nullptr, first.get(), slow.get());
    HYT_CUDA(cudaGetLastError());
    unsigned long long h_first = 0, h_slow = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_first, first.get(), 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaMemcpyAsync(&h_slow, slow.get(), 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    // 4. weights in other forms (exponents, many digits): the host parses
    //    those lines with the exact rules, from the same file
    int err_kind = 0;
    uint64_t err_line = ~uint64_t(0);
    if (h_first != ~0ull) {
        uint8_t k = 0;
        HYT_CUDA(cudaMemcpyAsync(&k, status.get() + h_first, 1, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        err_kind = k;
        err_line = h_first;
    }
    if (h_slow) {
        Scratch<uint8_t> flag(L, s);
        Scratch<uint64_t> idx(h_slow, s);
        slow_flags_kernel<<<grid_sm(8), 256, 0, s>>>(status.get(), L, flag.get());
        thrust::counting_iterator<uint64_t> it(0);
        size_t tb = 0;
        HYT_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flag.get(), idx.get(), nsel.get(), static_cast<int64_t>(L), s));
        Scratch<uint8_t> tmp(tb, s);
        HYT_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, it, flag.get(), idx.get(), nsel.get(), static_cast<int64_t>(L), s));
        Scratch<uint64_t> bb(h_slow, s), be(h_slow, s);
        line_bounds_kernel<<<grid_for(h_slow, 256), 256, 0, s>>>(ls.get(), L, size, idx.get(), h_slow, bb.get(), be.get());
        HYT_CUDA(cudaGetLastError());
        std::vector<uint64_t> hidx(h_slow), hb(h_slow), he(h_slow);
        HYT_CUDA(cudaMemcpyAsync(hidx.data(), idx.get(), h_slow * 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(hb.data(), bb.get(), h_slow * 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(he.data(), be.get(), h_slow * 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        void *m = ::mmap(nullptr, size, PROT_READ, MAP_PRIVATE, f.fd, 0);
        if (m == MAP_FAILED) fail(HYT_E_IO, "GraphLoader::load_edge_list: error while reading file: " + p);
        struct Unmap {
            void *m;
            uint64_t n;
            ~Unmap() { ::munmap(m, n); }
        } unmap{m, size};
        const char *ht = static_cast<const char *>(m);
        std::vector<uint8_t> hst(h_slow);
        std::vector<uint32_t> hs(h_slow), hd(h_slow), hw(h_slow);
        const unsigned T = host_threads(h_slow * 64, uint64_t(1) << 20);
        parallel_for(T, [&](unsigned t) {
            for (uint64_t k = h_slow * t / T, e = h_slow * (t + 1) / T; k < e; ++k)
                hst[k] = static_cast<uint8_t>(host_record(ht + hb[k], ht + he[k], V, weighted, hs[k], hd[k], hw[k]));
        });
        for (uint64_t k = 0; k < h_slow; ++k) {
            if (hst[k] >= kRecMalformed && hidx[k] < err_line) {
                err_line = hidx[k];
                err_kind = hst[k];
            }
        }
        Scratch<uint8_t> dst_(h_slow, s);
        Scratch<uint32_t> ds_(h_slow, s), dd_(h_slow, s), dw_(h_slow, s);
        HYT_CUDA(cudaMemcpyAsync(dst_.get(), hst.data(), h_slow, cudaMemcpyHostToDevice, s));
        HYT_CUDA(cudaMemcpyAsync(ds_.get(), hs.data(), h_slow * 4, cudaMemcpyHostToDevice, s));
        HYT_CUDA(cudaMemcpyAsync(dd_.get(), hd.data(), h_slow * 4, cudaMemcpyHostToDevice, s));
        HYT_CUDA(cudaMemcpyAsync(dw_.get(), hw.data(), h_slow * 4, cudaMemcpyHostToDevice, s));
        patch_lines_kernel<<<grid_for(h_slow, 256), 256, 0, s>>>(idx.get(), dst_.get(), ds_.get(), dd_.get(), dw_.get(),
                                                                 h_slow, status.get(), sv.get(), dv.get(),
                                                                 weighted ? wv->get() : nullptr);
        HYT_CUDA(cudaGetLastError());
        HYT_CUDA(cudaStreamSynchronize(s));
    }
    if (err_kind) {
        static const char *what[] = {"", "", "malformed edge", "vertex ID out of range", "missing edge weight",
                                     "unexpected data"};
        fail(HYT_E_INVALID, std::string("GraphLoader::load_edge_list: ") + what[err_kind] + " at line " +
                                std::to_string(err_line + 1));
    }
    // 5. the edges in file order
    Scratch<uint64_t> flag(L + 1, s), pos(L + 1, s);
    if (L) edge_flags_kernel<<<grid_sm(8), 256, 0, s>>>(status.get(), L, flag.get());
    HYT_CUDA(cudaMemsetAsync(flag.get() + L, 0, 8, s));
    {
        size_t tb = 0;
        HYT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.get(), pos.get(), static_cast<int64_t>(L + 1), s));
        Scratch<uint8_t> tmp(tb, s);
        HYT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, flag.get(), pos.get(), static_cast<int64_t>(L + 1), s));
    }
    uint64_t E = 0;
    HYT_CUDA(cudaMemcpyAsync(&E, pos.get() + L, 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    Scratch<uint32_t> cs(E, s), cd(E, s);
    std::unique_ptr<Scratch<uint32_t>> cw;
    if (weighted) cw = std::make_unique<Scratch<uint32_t>>(E, s);
    if (L)
        compact_edges_kernel<<<grid_sm(8), 256, 0, s>>>(status.get(), pos.get(), L, sv.get(), dv.get(),
                                                        weighted ? wv->get() : nullptr, cs.get(), cd.get(),
                                                        weighted ? cw->get() : nullptr);
    HYT_CUDA(cudaGetLastError());
    const double kms = build_csr(cs.get(), cd.get(), weighted ? cw->get() : nullptr, E, V,
                                 weighted ? HYT_WEIGHTS_F32 : HYT_WEIGHTS_NONE, on_device, out, s);
    whole.stop(s);
    if (stats) {
        stats->read_ms = read_ms;
        stats->device_ms = whole.ms();
        stats->kernel_ms = kms;
        stats->file_bytes = size;
        stats->num_edges = E;
        stats->kernel_bytes = construction_bytes(E, V, weighted);
        stats->threads = threads;
        stats->total_ms = ms_since(t0);
    }
}

void csr_save(const char *path, const hyt_csr &csr) {
    if (!path) fail(HYT_E_INVALID, "path is NULL");
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (V > (uint64_t(1) << 32)) fail(HYT_E_INVALID, "num_vertices must be at most 2^32 (32-bit vertex ids)");
    if (!csr.row_offsets || (E && !csr.column_indices)) fail(HYT_E_INVALID, "CSR arrays are NULL");
    if (csr.weight_kind != HYT_WEIGHTS_NONE && csr.weight_kind != HYT_WEIGHTS_U32 &&
        csr.weight_kind != HYT_WEIGHTS_F32)
        fail(HYT_E_INVALID, "unknown weight kind");
    const bool weighted = csr.weight_kind != HYT_WEIGHTS_NONE;
    if (weighted && E && !csr.weights) fail(HYT_E_INVALID, "weights are NULL");
    const Layout L(V, E, weighted);
    struct Sec {
        const void *p;
        uint64_t bytes, at;
    } secs[3] = {{csr.row_offsets, L.off_bytes, 0},
                 {csr.column_indices, L.cols_bytes, L.cols_at},
                 {weighted ? csr.weights : nullptr, L.w_bytes, L.w_at}};
    // checksum: device sections on the GPU, host sections on host threads;
    // the structure is checked the same way before anything is written
    StreamHold st;
    cudaStream_t s = st.s;
    uint64_t sum = 0;
    {
        Scratch<unsigned long long> dsum(1, s);
        HYT_CUDA(cudaMemsetAsync(dsum.get(), 0, 8, s));
        bool any_dev = false;
        for (const Sec &x : secs) {
            if (!x.p || !x.bytes) continue;
            if (is_device_pointer(x.p)) {
                any_dev = true;
                checksum_kernel<<<grid_for(x.bytes / 8 + 1, 256, 148u * 8u), 256, 0, s>>>(
                    static_cast<const uint32_t *>(x.p), x.bytes / 4, x.at / 8, dsum.get());
                HYT_CUDA(cudaGetLastError());
            } else {
                sum += host_checksum(static_cast<const uint32_t *>(x.p), x.bytes / 4, x.at / 8);
            }
        }
        if (any_dev) {
            unsigned long long h = 0;
            HYT_CUDA(cudaMemcpyAsync(&h, dsum.get(), 8, cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            sum += h;
        }
    }
    const bool dev_off = is_device_pointer(csr.row_offsets);
    const bool dev_cols = E && is_device_pointer(csr.column_indices);
    uint32_t bad = 0;
    if (dev_off || dev_cols) {
        std::unique_ptr<Scratch<uint64_t>> oh;
        std::unique_ptr<Scratch<uint32_t>> ch;
        const uint64_t *o = device_view(csr.row_offsets, V + 1, oh, s);
        const uint32_t *c = device_view(csr.column_indices, E, ch, s);
        Scratch<uint32_t> db(1, s);
        HYT_CUDA(cudaMemsetAsync(db.get(), 0, 4, s));
        check_structure_kernel<<<grid_for(std::max(V, E), 256, 148u * 8u), 256, 0, s>>>(o, c, V, E, db.get());
        HYT_CUDA(cudaGetLastError());
        HYT_CUDA(cudaMemcpyAsync(&bad, db.get(), 4, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
    } else {
        bad = host_structure(csr.row_offsets, csr.column_indices, V, E);
    }
    fail_structure(bad);
    FileHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.weight_kind = weighted ? csr.weight_kind : HYT_WEIGHTS_NONE;
    h.num_vertices = V;
    h.num_edges = E;
    h.payload_bytes = L.payload;
    h.checksum = sum;
    h.header_check = header_check(h);
    const std::string final_path(path);
    const std::string tmp = final_path + ".tmp." + std::to_string(::getpid());
    Fd f;
    f.fd = ::open(tmp.c_str(), O_CREAT | O_TRUNC | O_WRONLY, 0644);
    if (f.fd < 0) fail(HYT_E_IO, "unable to create file: " + tmp);
    try {
        write_all(f.fd, &h, sizeof(h), tmp);
        void *stage = nullptr;
        for (const Sec &x : secs) {
            if (!x.p || !x.bytes) continue;
            if (is_device_pointer(x.p)) {
                if (!stage) HYT_CUDA(cudaHostAlloc(&stage, kRingBytes, cudaHostAllocDefault));
                for (uint64_t d = 0; d < x.bytes; d += kRingBytes) {
                    const uint64_t n = std::min(kRingBytes, x.bytes - d);
                    HYT_CUDA(cudaMemcpyAsync(stage, static_cast<const char *>(x.p) + d, n, cudaMemcpyDeviceToHost, s));
                    HYT_CUDA(cudaStreamSynchronize(s));
                    write_all(f.fd, stage, n, tmp);
                }
            } else {
                write_all(f.fd, x.p, x.bytes, tmp);
            }
            const uint64_t zero = 0;
            if (pad8(x.bytes) != x.bytes) write_all(f.fd, &zero, pad8(x.bytes) - x.bytes, tmp);
        }
        if (stage) cudaFreeHost(stage);
        if (::close(f.fd) != 0) {
            f.fd = -1;
            fail(HYT_E_IO, "error while writing file: " + tmp);
        }
        f.fd = -1;
        if (::rename(tmp.c_str(), path) != 0) fail(HYT_E_IO, "unable to write file: " + final_path);
    } catch (...) {
        ::unlink(tmp.c_str());
        throw;
    }
}

void csr_load(const char *path, bool on_device, hyt_csr_buffers *out, hyt_load_stats *stats) {
    const auto t0 = Clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!out || !path) fail(HYT_E_INVALID, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    const std::string p(path);
    Fd f;
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) fail(HYT_E_IO, "unable to open file: " + p);
    struct stat sb {};
    if (::fstat(f.fd, &sb) != 0) fail(HYT_E_IO, "error while reading file: " + p);
    const uint64_t size = static_cast<uint64_t>(sb.st_size);
    if (size < sizeof(FileHeader)) fail(HYT_E_INVALID, "not a hytgraph CSR file (shorter than its header): " + p);
    FileHeader h{};
    read_all(f.fd, &h, sizeof(h), 0, "error while reading file: " + p);
    if (std::memcmp(h.magic, kMagic, 8) != 0) fail(HYT_E_INVALID, "not a hytgraph CSR file (bad magic): " + p);
    if (h.version != 1) fail(HYT_E_INVALID, "unsupported hytgraph CSR file version " + std::to_string(h.version));
    if (header_check(h) != h.header_check) fail(HYT_E_INVALID, "corrupt hytgraph CSR header: " + p);
    if (h.weight_kind > HYT_WEIGHTS_F32) fail(HYT_E_INVALID, "corrupt hytgraph CSR header (weight kind): " + p);
    const uint64_t V = h.num_vertices, E = h.num_edges;
    if (V > (uint64_t(1) << 32) || E > (uint64_t(1) << 40))
        fail(HYT_E_INVALID, "corrupt hytgraph CSR header (sizes): " + p);
    const bool weighted = h.weight_kind != HYT_WEIGHTS_NONE;
    const Layout L(V, E, weighted);
    if (L.payload != h.payload_bytes || size != sizeof(FileHeader) + L.payload)
        fail(HYT_E_INVALID, "file size does not match its header (truncated?): " + p);
    Output res(out, V, E, h.weight_kind, on_device);
    const uint64_t base = sizeof(FileHeader);
    std::vector<Piece> secs = {{base, reinterpret_cast<char *>(out->row_offsets), L.off_bytes},
                               {base + L.cols_at, reinterpret_cast<char *>(out->column_indices), L.cols_bytes}};
    if (weighted) secs.push_back({base + L.w_at, reinterpret_cast<char *>(out->weights), L.w_bytes});
    uint64_t sum = 0;
    uint32_t bad = 0;
    double read_ms = 0, dev_ms = 0, kms = 0;
    unsigned threads = 1;
    if (!on_device) {
        // every section cut into ranges, read by host threads
        std::vector<Piece> pieces;
        for (const Piece &x : secs)
            for (uint64_t d = 0; d < x.bytes; d += kRingBytes)
                pieces.push_back({x.file_at + d, x.dst + d, std::min(kRingBytes, x.bytes - d)});
        threads = host_threads(L.payload, kRingBytes);
        std::atomic<size_t> next{0};
        parallel_for(threads, [&](unsigned) {
            for (size_t k; (k = next.fetch_add(1)) < pieces.size();)
                read_all(f.fd, pieces[k].dst, pieces[k].bytes, pieces[k].file_at, "error while reading file: " + p);
        });
        read_ms = ms_since(t0);
        sum = host_checksum(reinterpret_cast<const uint32_t *>(out->row_offsets), L.off_bytes / 4, 0) +
              host_checksum(out->column_indices, E, L.cols_at / 8) +
              (weighted ? host_checksum(out->weights, E, L.w_at / 8) : 0);
        if (sum == h.checksum) bad = host_structure(out->row_offsets, out->column_indices, V, E);
    } else {
        std::vector<Piece> pieces;
        for (const Piece &x : secs) {
            const auto v = cut(x.file_at, x.dst, x.bytes);
            pieces.insert(pieces.end(), v.begin(), v.end());
        }
        const auto tr = Clock::now();
        threads = stream_to_device(f.fd, pieces, "error while reading file: " + p);
        read_ms = ms_since(tr);
        StreamHold st;
        cudaStream_t s = st.s;
        EventTimer whole;
        whole.start(s);
        Scratch<unsigned long long> dsum(1, s);
        Scratch<uint32_t> db(1, s);
        HYT_CUDA(cudaMemsetAsync(dsum.get(), 0, 8, s));
        HYT_CUDA(cudaMemsetAsync(db.get(), 0, 4, s));
        checksum_kernel<<<grid_for(L.off_bytes / 8 + 1, 256, 148u * 8u), 256, 0, s>>>(
            reinterpret_cast<const uint32_t *>(out->row_offsets), L.off_bytes / 4, 0, dsum.get());
        if (E)
            checksum_kernel<<<grid_for(E / 2 + 1, 256, 148u * 8u), 256, 0, s>>>(out->column_indices, E, L.cols_at / 8,
                                                                                dsum.get());
        if (weighted && E)
            checksum_kernel<<<grid_for(E / 2 + 1, 256, 148u * 8u), 256, 0, s>>>(out->weights, E, L.w_at / 8,
                                                                                dsum.get());
        check_structure_kernel<<<grid_for(std::max(V, E), 256, 148u * 8u), 256, 0, s>>>(
            out->row_offsets, out->column_indices, V, E, db.get());
        HYT_CUDA(cudaGetLastError());
        whole.stop(s);
        unsigned long long hs = 0;
        HYT_CUDA(cudaMemcpyAsync(&hs, dsum.get(), 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(&bad, db.get(), 4, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        sum = hs;
        kms = whole.ms();
        dev_ms = kms;
    }
    if (sum != h.checksum) fail(HYT_E_INVALID, "checksum mismatch: the file is corrupt: " + p);
    fail_structure(bad);
    res.armed = false;
    if (stats) {
        stats->read_ms = read_ms;
        stats->device_ms = dev_ms;
        stats->kernel_ms = kms;
        stats->file_bytes = size;
        stats->num_edges = E;
        // the checks read every payload byte once
        stats->kernel_bytes = L.off_bytes + L.cols_bytes + L.w_bytes;
        stats->threads = threads;
        stats->total_ms = ms_since(t0);
    }
}

}  // namespace hyt
