// rb2_trace_batch_noalloc: the batched traversal launch without any device
// allocation by the library.
//
// Who needs it: hosts that own every byte of device memory themselves -- a
// renderer or serving runtime that carves all device memory out of its own
// arena and admits work against a fixed budget, or a latency-critical loop in
// which cudaMalloc/cudaFree (which can synchronise the device and stall other
// streams) must not appear.  Those callers already hold the BVH, ray and
// output buffers in their own memory; what the regular batch path
// (rb2_batch_create) would allocate is only scratch: the job table, the
// ray-count prefix, the queue head and the status word.  Here that scratch is
// one file-scope __device__ array of fixed size (RB2_NOALLOC_MAX_JOBS jobs);
// every GPU that loads the library holds it until the process exits.
//
// Shared-state rules (also stated in include/rb2.h): every call reuses the
// same array, so two calls whose work overlaps on the GPU (different streams,
// or different host threads on the same device) race on it and corrupt each
// other's queue; serialise them on one stream.  The first call on a device
// resolves the array's device address (cudaGetSymbolAddress) and caches it;
// make that first call before any stream capture on that device.
#include "rb2.h"
#include "rb2_internal.h"
#include "rb2_sources.cuh"

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace {

// Scratch image: header words first (cleared by every call), then the prefix
// and the job table.  The host builds the same image on its stack and copies
// the used part in one transfer.
struct NoAllocScratch {
    unsigned long long counter;                         // queue head, starts at 0
    unsigned int status;                                // guard bits, start at 0
    unsigned int pad;
    unsigned long long start[RB2_NOALLOC_MAX_JOBS + 1]; // ray-count prefix
    alignas(16) rb2dev::JobDesc jobs[RB2_NOALLOC_MAX_JOBS];
};
static_assert(offsetof(NoAllocScratch, jobs) % 16 == 0, "job table alignment");

constexpr size_t kScratchWords = (sizeof(NoAllocScratch) + 7) / 8;

// The scratch array itself: ~18.5 KB per device.
static __device__ __align__(256) unsigned long long g_rb2_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;

struct DeviceSetup {
    bool ready = false;
    NoAllocScratch* scratch = nullptr;  // device address of g_rb2_noalloc_scratch
    int sms = 0;
    int ctas_per_sm = 0;
};

std::mutex g_setup_mu;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: resolve the array's device
// address and the launch shape.  Host code must never pass the symbol itself
// to a kernel -- in host code it names a host-side stand-in, not device memory.
int setup_current_device(DeviceSetup& out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return rb2::fail(RB2_ENOTSUP, "device ordinal beyond 63");
    std::lock_guard<std::mutex> g(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_rb2_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return rb2::fail(RB2_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        int sms = 0, per_sm = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("SM count: ") + cudaGetErrorString(e));
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, rb2dev::k_trace_jobs<128>, 128, rb2dev::job_smem_bytes(RB2_NOALLOC_MAX_JOBS, false));
        if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("occupancy: ") + cudaGetErrorString(e));
        s.scratch = static_cast<NoAllocScratch*>(p);
        s.sms = sms;
        s.ctas_per_sm = per_sm > 0 ? per_sm : 1;
        s.ready = true;
    }
    out = s;
    return RB2_OK;
}

}  // namespace

extern "C" int rb2_trace_batch_noalloc(const rb2_noalloc_job* jobs, uint32_t n_jobs, void* stream)
{
    if (n_jobs > RB2_NOALLOC_MAX_JOBS)
        return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: " + std::to_string(n_jobs) +
                                         " jobs exceed the fixed scratch capacity of " +
                                         std::to_string(RB2_NOALLOC_MAX_JOBS) + " jobs; split the batch");
    if (n_jobs && !jobs) return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: null job array");
    // Host image of the scratch, on the stack (no heap allocation either).
    NoAllocScratch img;
    img.counter = 0;
    img.status = 0;
    img.pad = 0;
    img.start[0] = 0;
    for (uint32_t i = 0; i < n_jobs; i++) {
        const rb2_noalloc_job& j = jobs[i];
        if (j.n && (!j.d_nodes || !j.d_woop || !j.d_triidx || !j.d_rays || !j.d_out))
            return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: job " + std::to_string(i) + " has a null buffer");
        if (j.mode > RB2_MODE_OCCLUSION) return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: unknown job mode");
        if (j.n > rb2dev::kMaxJobRays)
            return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: a job holds at most 2^32 - 1 rays");
        if (((uintptr_t)j.d_nodes | (uintptr_t)j.d_woop | (uintptr_t)j.d_rays) & 15u)
            return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: nodes, Woop rows and rays must be 16-byte aligned");
        if (j.mode != RB2_MODE_OCCLUSION && ((uintptr_t)j.d_out & 15u))
            return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc: hit records must be 16-byte aligned");
        rb2dev::JobDesc& d = img.jobs[i];
        d.nodes = reinterpret_cast<const float4*>(j.d_nodes);
        d.woop = reinterpret_cast<const float4*>(j.d_woop);
        d.triidx = j.d_triidx;
        d.rays = reinterpret_cast<const float4*>(j.d_rays);
        d.mask = j.d_mask;
        d.out = j.d_out;
        d.n = j.n;
        d.mode = j.mode;
        d.pad = 0;
        img.start[i + 1] = img.start[i] + j.n;
    }
    const unsigned long long total = img.start[n_jobs];
    if (total == 0) return RB2_OK;

    DeviceSetup dev;
    int rc = setup_current_device(dev);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // One copy clears the queue head and status and installs prefix + jobs.
    const size_t bytes = offsetof(NoAllocScratch, jobs) + sizeof(rb2dev::JobDesc) * n_jobs;
    cudaError_t e = cudaMemcpyAsync(dev.scratch, &img, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("scratch upload: ") + cudaGetErrorString(e));

    // Device addresses inside the scratch array (offset arithmetic only; the
    // host never dereferences them).
    char* base = reinterpret_cast<char*>(dev.scratch);
    rb2dev::KernelArgs a{};
    a.jobs = reinterpret_cast<const rb2dev::JobDesc*>(base + offsetof(NoAllocScratch, jobs));
    a.start = reinterpret_cast<const unsigned long long*>(base + offsetof(NoAllocScratch, start));
    a.n_jobs = n_jobs;
    a.fetch_threshold = 20;
    a.node_threshold = rb2dev::default_node_threshold(rb2dev::kLayoutBinary);
    a.chunk = 1;
    a.counter = reinterpret_cast<unsigned long long*>(base + offsetof(NoAllocScratch, counter));
    a.status = reinterpret_cast<unsigned int*>(base + offsetof(NoAllocScratch, status));
    uint64_t blocks = (uint64_t)dev.sms * (uint64_t)dev.ctas_per_sm;
    blocks = std::min<uint64_t>(blocks, (total + 127) / 128);
    blocks = std::max<uint64_t>(blocks, 1);
    rb2dev::k_trace_jobs<128><<<(unsigned)blocks, 128, rb2dev::job_smem_bytes(n_jobs, false), s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("trace launch: ") + cudaGetErrorString(e));
    return RB2_OK;
}

// Status of the last rb2_trace_batch_noalloc call on the current device: the
// guard bits its kernel set (bit 0: a ray's traversal stack would have
// overflowed, so that ray was reported as a miss).  The word is copied into
// the caller's host variable on `stream` and the stream is synchronised; no
// memory is allocated.  Same one-stream rule as the trace call: a query
// issued while another call's kernel is in flight on a different stream reads
// an unspecified value.
extern "C" int rb2_trace_batch_noalloc_status(uint32_t* status, void* stream)
{
    if (!status) return rb2::fail(RB2_EINVAL, "rb2_trace_batch_noalloc_status: null status pointer");
    DeviceSetup dev;
    int rc = setup_current_device(dev);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const char* base = reinterpret_cast<const char*>(dev.scratch);
    unsigned int word = 0;
    cudaError_t e = cudaMemcpyAsync(&word, base + offsetof(NoAllocScratch, status), sizeof(word),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return rb2::fail(RB2_ECUDA, std::string("status read: ") + cudaGetErrorString(e));
    *status = word;
    return RB2_OK;
}
