// Device allocations of librb2 go through these two wrappers so that a
// host-side fault injector (rb2_debug_fail_alloc) can make any one of them
// fail, and so that the library can count its live allocations
// (rb2_debug_alloc_count).  Injection happens on the host, before
// cudaMalloc is called: no GPU fault is involved.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>

namespace rb2 {

cudaError_t dev_malloc_bytes(void** p, size_t bytes);
cudaError_t dev_free(void* p);

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes)
{
    return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}

// RB2_ENOMEM for an allocation failure, RB2_ECUDA for any other CUDA error.
inline int cuda_status(cudaError_t e) { return e == cudaErrorMemoryAllocation ? 2 : 3; }

}  // namespace rb2
