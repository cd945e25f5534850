// Ray reordering for the batched traversal (rb2_batch_config.reorder).
//
// Each job's rays are visited in the order of a key: the ray's direction
// octant (3 bits, most significant) and a Morton code of its origin, k bits
// per axis (k = 3..6), within the job's scene box.  A counting sort builds the
// visiting order on the launch's stream (so it is captured in the batch's
// graph with the traversal).  The traversal then fetches ray perm[q] for queue
// slot q and writes its record to that ray's own index, so results do not
// depend on the order; only which rays share a warp does.
//
// The sort never uses global atomics.  The rays are cut into tiles that never
// cross a job (ReorderTile), and each pass over a digit of the key is:
//   1. count: one CTA per tile counts the digits of its entries in a
//      shared-memory histogram and stores it as its row of `cnt`
//      (tiles x buckets),
//   2. columns: per job and bucket, an exclusive scan down the job's tiles
//      turns each row into the tile's offset inside the bucket and leaves the
//      bucket's total in `tot` (jobs x buckets),
//   3. scan: an exclusive scan of `tot` in job-major order gives each
//      bucket's first position; job j's buckets land inside its own slot
//      range [start[j], start[j + 1]),
//   4. scatter: one CTA per tile loads its offsets into shared memory and
//      places each entry with a shared-memory atomic.
// For k <= 4 one pass sorts by the whole key (at most 2^15 buckets, whose
// counters fit in shared memory).  For k = 5, 6 a least-significant-digit
// sort of two passes: first by the low 3k - 12 Morton bits (entries become
// (key, slot) pairs), then by the high 15 bits (octant and the coarsest 12
// Morton bits) into perm.  The second pass keeps the first pass's order
// except inside a warp's 32 entries and among the entries that CTAs place
// concurrently, which share their low digit almost always; so the order is
// the key's up to such local swaps, which is all the traversal needs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rb2_sources.cuh"

namespace rb2 {

// A run of one job's entries: slots (or sorted positions) [begin, end), all in `job`.
struct ReorderTile {
    uint32_t job, begin, end, pad;
};

struct ReorderArgs {
    const rb2dev::JobDesc* jobs;            // device job table
    const unsigned long long* start;        // device prefix of job ray counts (n_jobs + 1)
    const float4* boxes;                    // per job: lo (xyz) and 1 / extent (xyz)
    uint32_t n_jobs;
    uint32_t bits;                          // k, 3..6
    uint64_t total;                         // rays in all jobs (< 2^32)
    const ReorderTile* tiles;               // n_tiles tiles, job-major, in slot order
    const uint32_t* job_tile0;              // n_jobs + 1: first tile of each job
    uint32_t* cnt;                          // n_tiles x buckets counters (per pass)
    uint32_t* tot;                          // n_jobs x buckets totals, then bucket starts
    uint32_t* chunk_sums;                   // scan scratch: one per 2048 totals
    uint32_t* keys;                         // total entries: each ray's key
    uint2* pairs;                           // total entries for k >= 5: (key, slot) after the first pass
    uint32_t* perm;                         // total entries: the visiting order
    uint32_t n_tiles;
};

constexpr uint32_t kReorderMinBits = 3, kReorderMaxBits = 6;
// Buckets of the high-digit pass of the two-pass sort (and the most of any pass).
constexpr uint32_t kReorderHighBits = 15;
// Widest key sorted in one pass.
constexpr uint32_t kReorderOnePassMaxBits = 4;

// Largest bucket count of any pass at k bits.
inline uint32_t reorder_max_buckets(uint32_t bits)
{
    return bits <= kReorderOnePassMaxBits ? 1u << (3 + 3 * bits) : 1u << kReorderHighBits;
}
inline uint64_t reorder_chunks(uint64_t counters) { return (counters + 2047) / 2048; }
// Rays per tile for a batch of `total` rays on `sms` SMs: about four tiles
// per SM, at least 8192 rays, a multiple of 1024.
inline uint32_t reorder_tile_rays(uint64_t total, int sms)
{
    const uint64_t per_sm = (uint64_t)(sms > 0 ? sms : 1) * 4;
    uint64_t t = (total + per_sm - 1) / per_sm;
    if (t < 8192) t = 8192;
    t = (t + 1023) / 1024 * 1024;
    return t > (1u << 30) ? (1u << 30) : (uint32_t)t;
}

// Lets the tile kernels use the shared memory of the widest histogram; call
// with the batch's device current before the first enqueue.
cudaError_t reorder_init();

// Enqueues the sort on `s`; returns a cudaError_t of the launches.
cudaError_t reorder_enqueue(const ReorderArgs& a, cudaStream_t s);

// Kernel launches of one sort at k bits (for launch accounting).
inline uint32_t reorder_launches(uint32_t bits) { return bits <= kReorderOnePassMaxBits ? 6u : 12u; }

}  // namespace rb2
