// Where an operand lives, seen from the GPU a handle was created on.
//
// Kept free of CUDA headers so that the rule can be compiled and checked on
// a machine without a GPU.  `memory_type` is a cudaMemoryType value as
// cudaPointerGetAttributes reports it (0 unregistered host memory, 1 pinned
// host memory, 2 device memory, 3 managed memory) and `pointer_device` that
// call's `device` field.
#pragma once

namespace iclb {

enum class MemKind {
    Host = 0,          // pinned (page-locked) host memory: staged by direct DMA
    Device = 1,        // the handle's GPU (or managed memory): used in place
    OtherDevice = 2,   // another GPU's memory: rejected (INVALID_VALUE)
    Pageable = 3,      // ordinary host memory: staged through pinned bounce buffers
};

inline MemKind classify_memory(int memory_type, int pointer_device, int handle_device)
{
    if (memory_type == 3) return MemKind::Device;
    if (memory_type == 2) return pointer_device == handle_device ? MemKind::Device : MemKind::OtherDevice;
    if (memory_type == 1) return MemKind::Host;
    return MemKind::Pageable;
}

}  // namespace iclb
