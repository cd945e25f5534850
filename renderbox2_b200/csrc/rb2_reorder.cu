// Ray reordering for the batched traversal: see rb2_reorder.cuh.
#include "rb2_reorder.cuh"

#include <algorithm>

namespace {

constexpr uint32_t kChunk = 2048;        // counters per scan chunk
constexpr uint32_t kThreads = 256;       // threads per scan block (8 counters each)
constexpr uint32_t kSmemJobs = 1024;     // job prefixes staged in shared memory up to this many jobs
constexpr uint32_t kTileThreads = 1024;  // threads per tile CTA of the tiled form

__device__ __forceinline__ uint32_t quantize(float x, float lo, float inv_extent, float cells, uint32_t qmax)
{
    const float q = (x - lo) * inv_extent * cells;
    // Origins outside the box (or NaN) clamp to its faces.
    if (!(q > 0.0f)) return 0u;
    return q >= (float)qmax ? qmax : (uint32_t)q;
}

// Key of a ray within its job: (direction octant, Morton code of the origin,
// k bits per axis), 3 + 3k bits.
__device__ __forceinline__ uint32_t key_of(const rb2::ReorderArgs& a, uint32_t j, uint64_t r)
{
    const rb2dev::JobDesc& d = a.jobs[j];
    const float4 o = __ldg(d.rays + 2 * r), dd = __ldg(d.rays + 2 * r + 1);
    const float4 lo = __ldg(a.boxes + 2 * (size_t)j), sc = __ldg(a.boxes + 2 * (size_t)j + 1);
    const uint32_t k = a.bits, qmax = (1u << k) - 1u;
    const float cells = (float)(1u << k);
    const uint32_t qx = quantize(o.x, lo.x, sc.x, cells, qmax), qy = quantize(o.y, lo.y, sc.y, cells, qmax),
                   qz = quantize(o.z, lo.z, sc.z, cells, qmax);
    uint32_t m = 0;
    for (uint32_t b = 0; b < k; b++)
        m |= (((qx >> b) & 1u) << (3 * b)) | (((qy >> b) & 1u) << (3 * b + 1)) | (((qz >> b) & 1u) << (3 * b + 2));
    const uint32_t oct = (dd.x < 0.0f ? 1u : 0u) | (dd.y < 0.0f ? 2u : 0u) | (dd.z < 0.0f ? 4u : 0u);
    return (oct << (3 * k)) | m;
}

// ---------------------------------------------------------------- tiled form

// Step 1: the tile's keys and its shared-memory histogram, stored as row t of cnt.
__global__ void __launch_bounds__(kTileThreads) k_tile_count(const rb2::ReorderArgs a)
{
    extern __shared__ uint32_t s_h[];
    const uint32_t nb = 1u << (3 + 3 * a.bits);
    for (uint32_t t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) s_h[i] = 0u;
        __syncthreads();
        const rb2::ReorderTile tl = a.tiles[t];
        const uint64_t s0 = a.start[tl.job];
        // Two rays per thread per pass, so each thread has both loads in flight.
        for (uint32_t s = tl.begin + threadIdx.x; s < tl.end; s += 2 * kTileThreads) {
            const uint32_t s2 = s + kTileThreads;
            const uint32_t k1 = key_of(a, tl.job, s - s0);
            const uint32_t k2 = s2 < tl.end ? key_of(a, tl.job, s2 - s0) : 0u;
            a.keys[s] = k1;
            atomicAdd(&s_h[k1], 1u);
            if (s2 < tl.end) {
                a.keys[s2] = k2;
                atomicAdd(&s_h[k2], 1u);
            }
        }
        __syncthreads();
        uint32_t* row = a.cnt + (uint64_t)t * nb;
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) row[i] = s_h[i];
        __syncthreads();
    }
}

// Step 2: per (job, bucket), an exclusive scan down the job's tiles, in place;
// the bucket's total goes to tot = a.hist.
__global__ void k_tile_columns(const rb2::ReorderArgs a)
{
    constexpr uint32_t kRows = 8;  // rows loaded together, so their loads overlap
    const uint32_t nb = 1u << (3 + 3 * a.bits);
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    uint32_t* __restrict__ cnt = a.cnt;
    for (uint32_t j = blockIdx.y; j < a.n_jobs; j += gridDim.y) {
        const uint32_t t0 = a.job_tile0[j], t1 = a.job_tile0[j + 1];
        uint32_t run = 0;
        for (uint32_t t = t0; t < t1; t += kRows) {
            const uint32_t m = t1 - t < kRows ? t1 - t : kRows;
            uint32_t c[kRows];
#pragma unroll
            for (uint32_t i = 0; i < kRows; i++) c[i] = i < m ? cnt[(uint64_t)(t + i) * nb + b] : 0u;
#pragma unroll
            for (uint32_t i = 0; i < kRows; i++) {
                if (i < m) cnt[(uint64_t)(t + i) * nb + b] = run;
                run += c[i];
            }
        }
        a.hist[(uint64_t)j * nb + b] = run;
    }
}

// Step 4: the tile's first position in every bucket (bucket start + the
// tile's offset inside it) in shared memory; each ray takes the next one.
__global__ void __launch_bounds__(kTileThreads) k_tile_scatter(const rb2::ReorderArgs a)
{
    extern __shared__ uint32_t s_off[];
    const uint32_t nb = 1u << (3 + 3 * a.bits);
    for (uint32_t t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const rb2::ReorderTile tl = a.tiles[t];
        const uint32_t* row = a.cnt + (uint64_t)t * nb;
        const uint32_t* base = a.hist + (uint64_t)tl.job * nb;
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) s_off[i] = base[i] + row[i];
        __syncthreads();
        for (uint32_t s = tl.begin + threadIdx.x; s < tl.end; s += kTileThreads) {
            const uint32_t pos = atomicAdd(&s_off[a.keys[s]], 1u);
            a.perm[pos] = s;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ global form (k = 5)

// Step 1 (kScatter false): each ray's key, kept in `keys`, and the bucket
// counts.  Step 3 (true): each ray takes the next position of its bucket,
// whose counter holds the bucket's start after the scan, and records its
// slot there.  Buckets are job-major: (job << (3 + 3k)) | key.
template <bool kScatter>
__global__ void k_reorder(const rb2::ReorderArgs a)
{
    extern __shared__ unsigned long long s_start[];
    const bool staged = a.n_jobs <= kSmemJobs;
    if (staged)
        for (uint32_t i = threadIdx.x; i <= a.n_jobs; i += blockDim.x) s_start[i] = a.start[i];
    __syncthreads();
    const unsigned long long* st = staged ? s_start : a.start;
    const uint32_t shift = 3 + 3 * a.bits;
    for (uint64_t slot = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; slot < a.total;
         slot += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = a.n_jobs;  // st[lo] <= slot < st[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (st[mid] <= slot) lo = mid; else hi = mid;
        }
        if constexpr (kScatter) {
            const uint64_t b = ((uint64_t)lo << shift) | a.keys[slot];
            const uint32_t pos = atomicAdd(&a.hist[b], 1u);
            a.perm[pos] = (uint32_t)slot;
        } else {
            const uint32_t key = key_of(a, lo, slot - st[lo]);
            a.keys[slot] = key;
            atomicAdd(&a.hist[((uint64_t)lo << shift) | key], 1u);
        }
    }
}

// ------------------------------------------------------------------- the scan

// Exclusive scan of the counters, in place (chunk sums, a scan of the sums in
// one block, then each chunk's own scan plus its offset).
__global__ void k_chunk_sums(const uint32_t* v, uint64_t n, uint32_t* sums)
{
    __shared__ uint32_t s_warp[kThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kChunk;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < kChunk; k += kThreads)
        if (base + k < n) c += v[base + k];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t w = 0; w < kThreads / 32; w++) t += s_warp[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void k_sums_scan(uint32_t* sums, uint32_t n)
{
    __shared__ uint32_t s[1024];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? sums[i] : 0u;
        s[threadIdx.x] = v;
        __syncthreads();
        for (uint32_t off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
            const uint32_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
            __syncthreads();
            s[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < n) sums[i] = carry + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += s[1023];
        __syncthreads();
    }
}

__global__ void k_chunk_scan(uint32_t* v, uint64_t n, const uint32_t* sums)
{
    __shared__ uint32_t s_warp[kThreads / 32];
    constexpr uint32_t kPer = kChunk / kThreads;   // consecutive counters per thread
    const uint64_t base = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kPer;
    uint32_t x[kPer];
    uint32_t t = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++) {
        x[k] = base + k < n ? v[base + k] : 0u;
        t += x[k];
    }
    // Exclusive prefix of the threads' totals within the block.
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = t;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t off = sums[blockIdx.x];
    for (uint32_t w = 0; w < warp; w++) off += s_warp[w];
    off += inc - t;
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++) {
        if (base + k < n) v[base + k] = off;
        off += x[k];
    }
}

cudaError_t scan_enqueue(uint32_t* v, uint64_t n, uint32_t* sums, cudaStream_t s)
{
    const uint64_t chunks = rb2::reorder_chunks(n);
    k_chunk_sums<<<(unsigned)chunks, kThreads, 0, s>>>(v, n, sums);
    k_sums_scan<<<1, 1024, 0, s>>>(sums, (uint32_t)chunks);
    k_chunk_scan<<<(unsigned)chunks, kThreads, 0, s>>>(v, n, sums);
    return cudaGetLastError();
}

}  // namespace

namespace rb2 {

cudaError_t reorder_init()
{
    const int smem = (int)(sizeof(uint32_t) << (3 + 3 * kReorderTiledMaxBits));
    cudaError_t e = cudaFuncSetAttribute(k_tile_count, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_tile_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

cudaError_t reorder_enqueue(const ReorderArgs& a, cudaStream_t s)
{
    if (a.total == 0) return cudaSuccess;
    const uint64_t buckets = reorder_buckets(a.n_jobs, a.bits);
    if (a.bits <= kReorderTiledMaxBits) {
        const uint32_t nb = (uint32_t)reorder_job_buckets(a.bits);
        const size_t smem = sizeof(uint32_t) * nb;
        k_tile_count<<<a.n_tiles, kTileThreads, smem, s>>>(a);
        const dim3 cols((nb + 255) / 256, std::min<uint32_t>(a.n_jobs, 65535u));
        k_tile_columns<<<cols, 256, 0, s>>>(a);
        cudaError_t e = scan_enqueue(a.hist, buckets, a.chunk_sums, s);
        if (e != cudaSuccess) return e;
        k_tile_scatter<<<a.n_tiles, kTileThreads, smem, s>>>(a);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(a.hist, 0, buckets * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const size_t smem = a.n_jobs <= kSmemJobs ? (a.n_jobs + 1) * sizeof(unsigned long long) : 0;
    const unsigned grid = (unsigned)std::min<uint64_t>((a.total + 255) / 256, (uint64_t)std::max(a.sms, 1) * 8);
    k_reorder<false><<<grid, 256, smem, s>>>(a);
    if ((e = scan_enqueue(a.hist, buckets, a.chunk_sums, s)) != cudaSuccess) return e;
    k_reorder<true><<<grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace rb2
