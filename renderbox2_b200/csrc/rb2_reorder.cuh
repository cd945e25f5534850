// Ray reordering for the batched traversal (rb2_batch_config.reorder).
//
// Each job's rays are visited in the order of a key: the ray's direction
// octant (3 bits, most significant) and a Morton code of its origin, k bits
// per axis, within the job's scene box.  A counting sort builds the visiting
// order on the launch's stream (so it is captured in the batch's graph with
// the traversal).  The traversal then fetches ray perm[q] for queue slot q and
// writes its record to that ray's own index, so results do not depend on the
// order; only which rays share a warp does.
//
// Two forms of the sort, by key width:
//
// k <= 4 (at most 2^15 buckets per job): tiled, with no global atomics.  The
// rays are cut into tiles that never cross a job (ReorderTile).
//   1. one CTA per tile computes each ray's key (kept in `keys`), counts the
//      keys in a shared-memory histogram and stores it as its row of
//      `cnt` (tiles x buckets),
//   2. per job and bucket, an exclusive scan down the job's tiles turns each
//      row into the tile's offset inside the bucket and leaves the bucket's
//      total in `tot` (jobs x buckets),
//   3. an exclusive scan of `tot` in job-major order gives each bucket's
//      first position; job j's buckets land inside its own slot range
//      [start[j], start[j + 1]),
//   4. one CTA per tile loads its offsets into shared memory and places each
//      of its rays with a shared-memory atomic (perm[position] = slot).
//
// k = 5 (2^18 buckets per job, too many for shared memory): the same three
// steps over one job-major bucket array with global atomics (counts, scan,
// scatter).
//
// In both forms the order within a bucket is whatever the atomics give.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rb2_sources.cuh"

namespace rb2 {

// A run of one job's rays: slots [begin, end) of the batch, all in `job`.
struct ReorderTile {
    uint32_t job, begin, end, pad;
};

struct ReorderArgs {
    const rb2dev::JobDesc* jobs;            // device job table
    const unsigned long long* start;        // device prefix of job ray counts (n_jobs + 1)
    const float4* boxes;                    // per job: lo (xyz) and 1 / extent (xyz)
    uint32_t n_jobs;
    uint32_t bits;                          // k, 3..5
    uint64_t total;                         // rays in all jobs (< 2^32)
    uint32_t* hist;                         // k = 5: n_jobs << (3 + 3k) counters; k <= 4: the per-job
                                            // bucket totals (`tot`, same size)
    uint32_t* chunk_sums;                   // scan scratch: one per 2048 counters
    uint32_t* keys;                         // total entries: each ray's key, count -> scatter
    uint32_t* perm;                         // total entries
    // tiled form (k <= 4)
    const ReorderTile* tiles;               // n_tiles tiles, job-major, in slot order
    const uint32_t* job_tile0;              // n_jobs + 1: first tile of each job
    uint32_t* cnt;                          // n_tiles << (3 + 3k) counters
    uint32_t n_tiles;
    int sms;
};

// Bucket counters per job at k bits.
inline uint64_t reorder_job_buckets(uint32_t bits) { return 1ull << (3 + 3 * bits); }
// Counters and chunk sums the reordering needs for n_jobs jobs at k bits.
inline uint64_t reorder_buckets(uint32_t n_jobs, uint32_t bits) { return (uint64_t)n_jobs << (3 + 3 * bits); }
inline uint64_t reorder_chunks(uint64_t buckets) { return (buckets + 2047) / 2048; }
// Widest key of the tiled form.
constexpr uint32_t kReorderTiledMaxBits = 4;
// Rays per tile of the tiled form for a batch of `total` rays on `sms` SMs:
// about four tiles per SM, at least 8192 rays, a multiple of 1024.
inline uint32_t reorder_tile_rays(uint64_t total, int sms)
{
    const uint64_t want = (total + (uint64_t)(sms > 0 ? sms : 1) * 4 - 1) / ((uint64_t)(sms > 0 ? sms : 1) * 4);
    uint64_t t = want < 8192 ? 8192 : want;
    t = (t + 1023) / 1024 * 1024;
    return t > (1u << 30) ? (1u << 30) : (uint32_t)t;
}

// Once per device: lets the tiled kernels use more than 48 KB of shared memory.
cudaError_t reorder_init();

// Enqueues the sort on `s`; returns a cudaError_t of the launches.
cudaError_t reorder_enqueue(const ReorderArgs& a, cudaStream_t s);

}  // namespace rb2
