// Shared helpers of the sm_100a core: status plumbing, device memory
// ownership, cache-policy loads and compensated (Kahan/TwoSum) arithmetic.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>

#include "hyt/capi.h"

namespace hyt {

// ---------------------------------------------------------------------------
// Status plumbing: internal code throws hyt::Error; every extern "C" entry
// point catches it, stores the message thread-locally and returns the code.
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);
void clear_last_error();

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? HYT_E_OOM
                         : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                             ? HYT_E_NO_DEVICE
                             : HYT_E_CUDA;
        (void)cudaGetLastError();  // clear a non-sticky error
        fail(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define HYT_CUDA(call) ::hyt::cuda_check((call), #call)

// Runs `body` and converts exceptions to a status code + thread-local message.
template <class F>
int guarded(F &&body) {
    try {
        clear_last_error();
        body();
        return HYT_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return HYT_E_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return HYT_E_INTERNAL;
    }
}

// ---------------------------------------------------------------------------
// Owning device buffer (cudaMalloc / cudaFree), move-only.
// ---------------------------------------------------------------------------
template <class T>
struct DeviceArray {
    T *ptr = nullptr;
    size_t count = 0;

    DeviceArray() = default;
    explicit DeviceArray(size_t n) { allocate(n); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : ptr(o.ptr), count(o.count) { o.ptr = nullptr; o.count = 0; }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; count = o.count; o.ptr = nullptr; o.count = 0; }
        return *this;
    }
    ~DeviceArray() { release(); }

    void allocate(size_t n) {
        release();
        if (n == 0) return;
        // 16 bytes of tail padding so vectorised / bulk loads of the last
        // elements never touch memory outside the allocation.
        void *p = nullptr;
        HYT_CUDA(cudaMalloc(&p, n * sizeof(T) + 16));
        ptr = static_cast<T *>(p);
        count = n;
    }
    void release() noexcept {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
    T *get() const { return ptr; }
};

// Device pool for long-lived graph arrays: stream-ordered allocations from
// one pool per device that keeps up to kGraphPoolKeep bytes mapped after
// they are freed, so creating and destroying graphs repeatedly does not pay
// for mapping fresh memory each time (hyt_trim_device_memory returns it).
constexpr uint64_t kGraphPoolKeep = uint64_t(16) << 30;
cudaMemPool_t graph_pool(int device);

// Owning device buffer from the graph pool; same interface as DeviceArray.
// Allocation completes before allocate() returns; release() waits for the
// device (as cudaFree does) before handing the memory back.
template <class T>
struct GraphArray {
    T *ptr = nullptr;
    size_t count = 0;
    int dev = 0;

    GraphArray() = default;
    explicit GraphArray(size_t n) { allocate(n); }
    GraphArray(const GraphArray &) = delete;
    GraphArray &operator=(const GraphArray &) = delete;
    GraphArray(GraphArray &&o) noexcept : ptr(o.ptr), count(o.count), dev(o.dev) { o.ptr = nullptr; o.count = 0; }
    GraphArray &operator=(GraphArray &&o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            count = o.count;
            dev = o.dev;
            o.ptr = nullptr;
            o.count = 0;
        }
        return *this;
    }
    ~GraphArray() { release(); }

    void allocate(size_t n) {
        release();
        if (n == 0) return;
        HYT_CUDA(cudaGetDevice(&dev));
        void *p = nullptr;
        // 16 bytes of tail padding, as DeviceArray
        HYT_CUDA(cudaMallocFromPoolAsync(&p, n * sizeof(T) + 16, graph_pool(dev), cudaStreamLegacy));
        HYT_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
        ptr = static_cast<T *>(p);
        count = n;
    }
    void release() noexcept {
        if (ptr) {
            int cur = 0;
            cudaGetDevice(&cur);
            if (cur != dev) cudaSetDevice(dev);
            cudaDeviceSynchronize();  // no kernel may still use it
            cudaFreeAsync(ptr, cudaStreamLegacy);
            cudaStreamSynchronize(cudaStreamLegacy);
            if (cur != dev) cudaSetDevice(cur);
        }
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
    T *get() const { return ptr; }
};

// Owning pinned host buffer.
template <class T>
struct PinnedArray {
    T *ptr = nullptr;
    size_t count = 0;
    PinnedArray() = default;
    explicit PinnedArray(size_t n, unsigned flags = cudaHostAllocDefault) { allocate(n, flags); }
    PinnedArray(const PinnedArray &) = delete;
    PinnedArray &operator=(const PinnedArray &) = delete;
    ~PinnedArray() { release(); }
    void allocate(size_t n, unsigned flags = cudaHostAllocDefault) {
        release();
        if (n == 0) return;
        void *p = nullptr;
        HYT_CUDA(cudaHostAlloc(&p, n * sizeof(T), flags));
        ptr = static_cast<T *>(p);
        count = n;
    }
    void release() noexcept {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        count = 0;
    }
};

// True when `p` is device (or managed) memory on some GPU.
bool is_device_pointer(const void *p);

enum class PointerPlace;
// Where `p` lives relative to `current_device` (host_checks.hpp);
// *pointer_device receives the ordinal cudaPointerGetAttributes reports
// (-1 when it reports none).
PointerPlace pointer_place(const void *p, int current_device, int *pointer_device);

// Copies `bytes` from src (host or device) into device memory dst.
void copy_to_device(void *dst, const void *src, size_t bytes, cudaStream_t s);
// Copies `bytes` from device memory src into dst (host or device).
void copy_from_device(void *dst, const void *src, size_t bytes, cudaStream_t s);

// RAII CUDA event pair for device timing on one stream.
struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    EventTimer() {
        HYT_CUDA(cudaEventCreate(&a));
        HYT_CUDA(cudaEventCreate(&b));
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { HYT_CUDA(cudaEventRecord(a, s)); }
    void stop(cudaStream_t s) { HYT_CUDA(cudaEventRecord(b, s)); }
    double ms() {
        HYT_CUDA(cudaEventSynchronize(b));
        float t = 0.f;
        HYT_CUDA(cudaEventElapsedTime(&t, a, b));
        return static_cast<double>(t);
    }
};

int sm_count();

// A negative device ordinal in creation options selects the calling
// thread's current device.
inline int resolve_device(int device) {
    if (device >= 0) return device;
    int cur = 0;
    HYT_CUDA(cudaGetDevice(&cur));
    return cur;
}

inline unsigned grid_for(size_t n, unsigned block, unsigned cap = 148u * 32u) {
    size_t g = (n + block - 1) / block;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return static_cast<unsigned>(g);
}

}  // namespace hyt

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__

namespace hyt::dev {

// Streaming load: the edge arrays are read once per pass; evict-first keeps
// them from displacing the L2-resident vertex arrays.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }
__device__ __forceinline__ uint4 ld_stream4(const uint4 *p) { return __ldcs(p); }
__device__ __forceinline__ uint64_t ld_stream(const uint64_t *p) {
    return __ldcs(reinterpret_cast<const unsigned long long *>(p));
}

// Gather through L2 with an evict-last policy: per-vertex arrays (ranks,
// contributions, distances) are reused across the whole pass.
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_keep(const float *p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

// Coherent 32-bit load with an L2 cache-eviction policy (for data other
// threads may update during the kernel).
__device__ __forceinline__ uint32_t ld_keep_u32(const uint32_t *p, uint64_t pol) {
    uint32_t v;
    asm volatile("ld.global.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// Error-free transformation (Knuth TwoSum): a + b = s + e exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

// Compensated accumulator: Kahan summation per element (4 adds; c holds
// the negated low-order part, value = s - c), TwoSum when two partial sums
// merge (warp reductions, long-row chunks).
struct CSum {
    float s = 0.f;
    float c = 0.f;
    __device__ __forceinline__ void add(float x) {
        const float y = __fsub_rn(x, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ void merge(const CSum &o) {
        float t, e;
        two_sum(s, o.s, t, e);  // s + o.s = t + e exactly
        s = t;
        c = __fsub_rn(__fadd_rn(c, o.c), e);
    }
    __device__ __forceinline__ float value() const { return __fsub_rn(s, c); }
};

__device__ __forceinline__ CSum warp_reduce(CSum v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        CSum w;
        w.s = __shfl_xor_sync(0xffffffffu, v.s, o);
        w.c = __shfl_xor_sync(0xffffffffu, v.c, o);
        v.merge(w);
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide FP64 sum; result valid in thread 0.  `scratch` holds >= 32.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
    if (warp == 0) v = warp_sum(v);
    return v;
}

}  // namespace hyt::dev

#endif  // __CUDACC__
