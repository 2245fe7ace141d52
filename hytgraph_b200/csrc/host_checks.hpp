// Host-side decisions of the C ABI that need no GPU to evaluate: the
// default creation options and where a caller's pointer lives.  Kept free of
// CUDA calls so CPU unit tests can exercise them with made-up inputs.
#pragma once

#include <driver_types.h>

namespace hyt {

// The creation options the caller passed, or -- for NULL -- all zeros except
// the device ordinal, which is -1: the calling thread's current device.  A
// process that drives one GPU (one process per GPU) thus keeps every handle
// on its own GPU without naming the ordinal, and its current device is left
// as it was.
template <class Options>
Options options_or_default(const Options *given) {
    if (given) return *given;
    Options o{};
    o.device = -1;
    return o;
}

// Where a pointer lives, from the memory type and device ordinal that
// cudaPointerGetAttributes reports for it.
enum class PointerPlace {
    kCurrentDevice,  // device memory of the current device, or managed memory
    kOtherDevice,    // device memory of another GPU: unreachable without peer access
    kHost            // pageable, pinned or unknown host memory
};

inline PointerPlace classify_pointer(cudaMemoryType type, int pointer_device, int current_device) {
    if (type == cudaMemoryTypeManaged) return PointerPlace::kCurrentDevice;
    if (type == cudaMemoryTypeDevice)
        return pointer_device == current_device ? PointerPlace::kCurrentDevice : PointerPlace::kOtherDevice;
    return PointerPlace::kHost;
}

}  // namespace hyt
