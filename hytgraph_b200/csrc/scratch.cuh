// Stream-ordered scratch memory and small host helpers shared by the
// one-shot graph transforms (hub sort, reorder, CSR construction, loading).
#pragma once

#include <algorithm>
#include <memory>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace hyt {

// Scratch pool of the current device: stream-ordered allocations that keep
// up to 8 GiB mapped between calls, so repeated calls do not pay for
// mapping fresh memory (building a scale-24 graph needs a few GB of
// temporaries; hyt_trim_device_memory returns them).
inline cudaMemPool_t scratch_pool() {
    static std::mutex mu;
    static std::unordered_map<int, cudaMemPool_t> pools;
    int dev = 0;
    HYT_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    HYT_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = uint64_t(8) << 30;
    HYT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
    return pool;
}

// Stream-ordered scratch (freed on the same stream at scope exit).
template <class T>
struct Scratch {
    T *p = nullptr;
    cudaStream_t s = nullptr;
    Scratch(size_t n, cudaStream_t st) : s(st) {
        void *q = nullptr;
        HYT_CUDA(cudaMallocFromPoolAsync(&q, std::max<size_t>(n, 1) * sizeof(T) + 16, scratch_pool(), s));
        p = static_cast<T *>(q);
    }
    ~Scratch() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    T *get() const { return p; }
};

// Device view of a host-or-device array: device pointers pass through, host
// arrays are copied into `hold`.
template <class T>
const T *device_view(const T *p, uint64_t n, std::unique_ptr<Scratch<T>> &hold, cudaStream_t s) {
    if (!p || n == 0 || is_device_pointer(p)) return p;
    hold = std::make_unique<Scratch<T>>(n, s);
    HYT_CUDA(cudaMemcpyAsync(hold->get(), p, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return hold->get();
}

struct StreamHold {
    cudaStream_t s = nullptr;
    StreamHold() { HYT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~StreamHold() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

}  // namespace hyt
