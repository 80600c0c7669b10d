// Which caller arrays a kernel launched on the current device may read and write: device
// memory of that same device, or managed memory (migrates on access). Host memory, unregistered
// memory and another GPU's device memory are refused (without peer access a kernel that
// touched them would fault). Kept free of CUDA headers so that a host-only test can check it;
// the memory-type values are those of cudaMemoryType (checked where it is used).
#pragma once

namespace cfdb {

enum PointerType : int { kPtrUnregistered = 0, kPtrHost = 1, kPtrDevice = 2, kPtrManaged = 3 };

inline bool pointer_usable_on(int memory_type, int pointer_device, int current_device) {
    if (memory_type == kPtrDevice) return pointer_device == current_device;
    return memory_type == kPtrManaged;
}

} // namespace cfdb
