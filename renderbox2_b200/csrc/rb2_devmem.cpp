// Device allocation wrappers and the allocation fault injector (rb2_devmem.h).
#include "rb2_devmem.h"

#include "rb2.h"
#include "rb2_internal.h"

#include <atomic>

namespace {

std::atomic<uint64_t> g_allocs{0};       // successful allocations since load
std::atomic<int64_t> g_live{0};          // allocations not yet freed
std::atomic<uint64_t> g_fail_at{0};      // 0: off; k: the k-th allocation from arming fails
std::atomic<uint64_t> g_since_arm{0};

}  // namespace

namespace rb2 {

cudaError_t dev_malloc_bytes(void** p, size_t bytes)
{
    const uint64_t k = g_fail_at.load();
    if (k) {
        const uint64_t n = ++g_since_arm;
        if (n == k) {
            g_fail_at.store(0);
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) *p = nullptr;
    if (e == cudaSuccess && *p) {
        ++g_allocs;
        ++g_live;
    }
    return e;
}

cudaError_t dev_free(void* p)
{
    if (!p) return cudaSuccess;
    cudaError_t e = cudaFree(p);
    if (e == cudaSuccess) --g_live;
    return e;
}

}  // namespace rb2

extern "C" int rb2_debug_fail_alloc(uint64_t k)
{
    g_since_arm.store(0);
    g_fail_at.store(k);
    return RB2_OK;
}

extern "C" int rb2_debug_alloc_count(uint64_t* total, int64_t* live)
{
    if (total) *total = g_allocs.load();
    if (live) *live = g_live.load();
    return RB2_OK;
}
