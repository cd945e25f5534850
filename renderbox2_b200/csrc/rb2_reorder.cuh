// Ray reordering for the batched traversal (rb2_batch_config.reorder).
//
// Each job's rays are visited in the order of a key: the ray's direction
// octant (3 bits, most significant) and a Morton code of its origin, k bits
// per axis, within the job's scene box.  A counting sort builds the visiting
// order in three stages on the launch's stream (so it is captured in the
// batch's graph with the traversal):
//   1. each ray's key (kept for stage 3, so rays are read once) and per
//      (job, key) bucket counts (atomics),
//   2. an exclusive scan of the job-major bucket array, which places job j's
//      buckets inside its own slot range [start[j], start[j + 1]),
//   3. a scatter: each ray takes the next position of its bucket and writes
//      its slot there (perm[position] = slot); the order within a bucket is
//      whatever the atomics give.
// The traversal then fetches ray perm[q] for queue slot q and writes its
// record to that ray's own index, so results do not depend on the order;
// only which rays share a warp does.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rb2_sources.cuh"

namespace rb2 {

struct ReorderArgs {
    const rb2dev::JobDesc* jobs;            // device job table
    const unsigned long long* start;        // device prefix of job ray counts (n_jobs + 1)
    const float4* boxes;                    // per job: lo (xyz) and 1 / extent (xyz)
    uint32_t n_jobs;
    uint32_t bits;                          // k, 3..5
    uint64_t total;                         // rays in all jobs (< 2^32)
    uint32_t* hist;                         // n_jobs << (3 + 3k) counters
    uint32_t* chunk_sums;                   // scan scratch: one per 2048 counters
    uint32_t* keys;                         // total entries: each ray's key, stage 1 -> stage 3
    uint32_t* perm;                         // total entries
    int sms;
};

// Counters and chunk sums the reordering needs for n_jobs jobs at k bits.
inline uint64_t reorder_buckets(uint32_t n_jobs, uint32_t bits) { return (uint64_t)n_jobs << (3 + 3 * bits); }
inline uint64_t reorder_chunks(uint64_t buckets) { return (buckets + 2047) / 2048; }

// Enqueues the three stages on `s`; returns a cudaError_t of the launches.
cudaError_t reorder_enqueue(const ReorderArgs& a, cudaStream_t s);

}  // namespace rb2
