// hj_workspace.h -- a device workspace lent to a thread's temporaries (plain
// C++, shared by the CUDA sources and the host-only serving loop).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace hj {

// A device workspace a thread lends to the Scratch guards it runs (the serving
// loop gives each worker one): temporaries are carved from its top like a stack
// and given back when their guard ends, so a small request's temporaries cost
// no allocator calls.  Only the innermost live guard on the workspace's own
// stream takes from it; everything else, and whatever does not fit, comes from
// the memory pool.
struct Workspace {
    char* base = nullptr;
    size_t cap = 0;
    size_t top = 0;
    uint32_t depth = 0;           // live guards
    cudaStream_t stream = nullptr;
};
Workspace* current_workspace();            // hj_index.cu (per thread)
void set_current_workspace(Workspace* ws);

}  // namespace hj
