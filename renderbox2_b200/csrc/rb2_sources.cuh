// Job-table ray source for persistent_trace (rb2_traverse.cuh) and the one
// traversal kernel template every launch uses: a single-scene trace is a job
// table of one entry passed inline in the kernel parameters; a batched launch
// reads up to any number of (scene BVH, ray batch, mode) jobs from device
// memory and serves all of them from one global queue.
#pragma once

#include "rb2_traverse.cuh"
#include "rb2_traverse_cw8.cuh"

namespace rb2dev {

// Job descriptor (64 bytes): one scene's BVH plus one ray batch.
struct JobDesc {
    const float4* nodes;
    const float4* woop;
    const uint32_t* triidx;
    const float4* rays;     // 2 float4 per ray
    const uint8_t* mask;    // nullable stencil
    void* out;              // int4 hit records (modes 0/1) or uint8 occlusion (mode 2)
    uint64_t n;
    uint32_t mode;
    uint32_t pad;
};
static_assert(sizeof(JobDesc) == 64, "job descriptor layout");

constexpr uint32_t kMaxSmemJobs = 1024;


struct KernelArgs {
    const JobDesc* jobs;                 // nullptr: use inline_job (n_jobs == 1)
    const unsigned long long* start;     // n_jobs + 1 prefix offsets of the jobs' rays
    JobDesc inline_job;
    uint32_t n_jobs;
    uint32_t fetch_threshold;            // refill a warp when fewer lanes stay busy
    uint32_t chunk;                      // warp reserves chunk*32 slots per atomic (<= 1: exact)
    uint32_t node_threshold;             // end a node phase below this many lanes (persistent_trace*)
    unsigned long long* counter;         // queue head (zeroed before the launch)
    unsigned int* status;                // guard bits
    const uint32_t* perm;                // nullable: queue slot -> ray slot (ray reordering)
};

struct JobSource {
    const JobDesc* jobs;
    const unsigned long long* start;
    uint32_t n_jobs;
    unsigned long long total;
    unsigned long long* counter;
    uint32_t chunk;
    unsigned long long* rem;             // per-warp private [cur, end) in shared memory
    const uint32_t* perm;                // nullable: the order in which ray slots are visited

    __device__ __forceinline__ void claim(unsigned count, unsigned long long& b1, unsigned& n1,
                                          unsigned long long& b2)
    {
        if (chunk <= 1) {
            b1 = atomicAdd(counter, (unsigned long long)count);
            n1 = count;
            b2 = 0;
            return;
        }
        unsigned long long* r = rem + 2 * (threadIdx.x >> 5);
        const unsigned long long cur = r[0], end = r[1], avail = end - cur;
        if (avail >= count) {
            b1 = cur; n1 = count; b2 = 0;
            r[0] = cur + count;
            return;
        }
        const unsigned long long size = (unsigned long long)chunk * 32ull;
        const unsigned long long fresh = atomicAdd(counter, size);
        b1 = cur; n1 = (unsigned)avail; b2 = fresh;
        r[0] = fresh + (count - n1);
        r[1] = fresh + size;
    }

    __device__ __forceinline__ uint32_t find_job(unsigned long long slot) const
    {
        uint32_t lo = 0, hi = n_jobs;  // start[lo] <= slot < start[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (start[mid] <= slot) lo = mid; else hi = mid;
        }
        return lo;
    }

    __device__ __forceinline__ int fetch(unsigned long long slot, Lane& L) const
    {
        if (slot >= total) return 0;
        if (perm != nullptr) slot = __ldg(perm + slot);  // a permutation of [0, total), job ranges kept
        const uint32_t j = find_job(slot);
        const JobDesc& d = jobs[j];
        const uint64_t r = slot - start[j];
        L.set_tag(d.mode, j);
        L.ray = (uint32_t)r;
        if (d.mask != nullptr && d.mask[r] == 0) {
            const float4 d4 = __ldg(d.rays + 2 * r + 1);
            if (d.mode == kOcclusion) static_cast<uint8_t*>(d.out)[r] = 0;
            else static_cast<int4*>(d.out)[r] = make_int4(-1, __float_as_int(d4.w), 0, 0);
            return -1;
        }
        L.nodes = d.nodes;
        L.woop = d.woop;
        setup_ray(L, __ldg(d.rays + 2 * r), __ldg(d.rays + 2 * r + 1));
        return 1;
    }

    __device__ __forceinline__ void finish(const Lane& L) const
    {
        const JobDesc& d = jobs[L.job()];
        if (L.mode() == kOcclusion) static_cast<uint8_t*>(d.out)[L.ray] = L.hitIndex >= 0 ? 1 : 0;
        else static_cast<int4*>(d.out)[L.ray] = hit_record(L, d.triidx);
    }
};

// Dynamic shared memory holds the job prefix table (n_jobs + 1 entries, or 2
// for an inline job) so small batches leave the rest of the SM's 256 KB for L1.
__host__ __device__ constexpr size_t job_smem_bytes(uint32_t n_jobs, bool inline_job)
{
    return inline_job ? 2 * sizeof(unsigned long long)
                      : (n_jobs <= kMaxSmemJobs ? (n_jobs + 1) * sizeof(unsigned long long) : 0);
}

// REGS is the register budget per thread the variant is compiled for (64:
// 32 resident warps per SM, 48: 40 warps, 40: 48 warps; lower budgets spill a
// little state to L1).  The autotuner picks the variant by measurement.
// LAYOUT: what the jobs' node buffers hold: kLayoutBinary (Compact2),
// kLayoutWide4 (kWideEmpty, rb2_traverse.cuh) or kLayoutCw8 (rb2_traverse_cw8.cuh).
template <int BLOCK, int REGS = 64, int LAYOUT = kLayoutBinary>
__global__ void __launch_bounds__(BLOCK, (65536 / REGS) / BLOCK) k_trace_jobs(const __grid_constant__ KernelArgs a)
{
    extern __shared__ unsigned long long s_start[];
    __shared__ unsigned long long s_rem[2 * (BLOCK / 32)];
    __shared__ JobDesc s_job;
    const uint32_t nj = a.n_jobs;
    const bool inline_job = a.jobs == nullptr;
    const bool smem_start = inline_job || nj <= kMaxSmemJobs;
    if (inline_job) {
        if (threadIdx.x == 0) {
            s_job = a.inline_job;
            s_start[0] = 0;
            s_start[1] = a.inline_job.n;
        }
    } else if (smem_start) {
        for (uint32_t i = threadIdx.x; i <= nj; i += BLOCK) s_start[i] = a.start[i];
    }
    if (threadIdx.x < 2 * (BLOCK / 32)) s_rem[threadIdx.x] = 0;
    __syncthreads();

    JobSource src;
    src.jobs = inline_job ? &s_job : a.jobs;
    src.start = smem_start ? s_start : a.start;
    src.n_jobs = inline_job ? 1u : nj;
    src.total = src.start[src.n_jobs];
    src.counter = a.counter;
    src.chunk = a.chunk;
    src.rem = s_rem;
    src.perm = a.perm;
    if constexpr (LAYOUT == kLayoutCw8) persistent_trace_cw8<JobSource>(src, a.fetch_threshold, a.node_threshold, a.status);
    else persistent_trace<JobSource, LAYOUT == kLayoutWide4>(src, a.fetch_threshold, a.node_threshold, a.status);
}

}  // namespace rb2dev
