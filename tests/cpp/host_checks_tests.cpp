// CPU tests of the C ABI's host-side decisions (hytgraph_b200/csrc/
// host_checks.hpp) with made-up inputs: no GPU is needed or touched.
//   - NULL creation options mean the calling thread's current device
//     (device ordinal -1) for graphs, hybrids, batches and servers;
//   - hyt_sssp_noalloc's pointer test refuses host memory and the device
//     memory of another GPU, and accepts the current GPU's and managed memory.
#include <cstdio>
#include <cstdlib>

#include "host_checks.hpp"
#include "hyt/capi.h"

static int failures = 0;
#define CHECK(cond)                                                       \
    do {                                                                  \
        if (!(cond)) {                                                    \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                   \
        }                                                                 \
    } while (0)

template <class O>
static void null_means_current_device() {
    const O d = hyt::options_or_default<O>(nullptr);
    CHECK(d.device == -1);
    O given{};
    given.device = 3;
    CHECK(hyt::options_or_default(&given).device == 3);
    given.device = 0;
    CHECK(hyt::options_or_default(&given).device == 0);
}

int main() {
    null_means_current_device<hyt_graph_options>();
    null_means_current_device<hyt_hybrid_options>();
    null_means_current_device<hyt_batch_options>();
    null_means_current_device<hyt_server_options>();
    {
        const hyt_graph_options d = hyt::options_or_default<hyt_graph_options>(nullptr);
        CHECK(d.flags == 0 && d.stream == nullptr);
    }
    using hyt::PointerPlace;
    using hyt::classify_pointer;
    CHECK(classify_pointer(cudaMemoryTypeDevice, 0, 0) == PointerPlace::kCurrentDevice);
    CHECK(classify_pointer(cudaMemoryTypeDevice, 5, 5) == PointerPlace::kCurrentDevice);
    CHECK(classify_pointer(cudaMemoryTypeDevice, 1, 0) == PointerPlace::kOtherDevice);
    CHECK(classify_pointer(cudaMemoryTypeDevice, 0, 7) == PointerPlace::kOtherDevice);
    CHECK(classify_pointer(cudaMemoryTypeManaged, 2, 0) == PointerPlace::kCurrentDevice);
    CHECK(classify_pointer(cudaMemoryTypeHost, 0, 0) == PointerPlace::kHost);
    CHECK(classify_pointer(cudaMemoryTypeUnregistered, -1, 0) == PointerPlace::kHost);
    if (failures) return 1;
    std::printf("host checks passed\n");
    return 0;
}
