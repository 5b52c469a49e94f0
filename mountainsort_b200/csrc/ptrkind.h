// Where a caller's buffer lives, decided from the fields that
// cudaPointerGetAttributes reports.  Kept free of CUDA headers so the rule
// can be checked on a machine without a GPU.
#pragma once

namespace ms3gpu {

enum class PtrKind {
    Host,             // pageable or pinned host memory: staged through the device
    DeviceHere,       // device memory of the current device: used in place
    Managed,          // managed memory: reachable from every device, used in place
    DeviceElsewhere,  // device memory of another GPU: rejected
};

// type: the cudaMemoryType value (0 unregistered, 1 host, 2 device,
// 3 managed); device: the attribute's device ordinal; current: the device the
// call runs on.
inline PtrKind classify_pointer(int type, int device, int current) {
    switch (type) {
    case 2:
        return device == current ? PtrKind::DeviceHere : PtrKind::DeviceElsewhere;
    case 3:
        return PtrKind::Managed;
    default:
        return PtrKind::Host;
    }
}

}  // namespace ms3gpu
