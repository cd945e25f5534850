// Ray reordering for the batched traversal: see rb2_reorder.cuh.
#include "rb2_reorder.cuh"

#include <algorithm>

namespace {

constexpr uint32_t kChunk = 2048;        // counters per scan chunk
constexpr uint32_t kThreads = 256;       // threads per scan block (8 counters each)
constexpr uint32_t kTileThreads = 1024;  // threads per tile CTA
constexpr uint32_t kWarpAggMax = 64;     // histograms this small aggregate each warp's equal digits

// Passes of the sort: the whole key (k <= 4), or the low then the high digit (k = 5, 6).
enum Pass : int { kWhole = 0, kLow = 1, kHigh = 2 };

__device__ __forceinline__ uint32_t low_bits(uint32_t k) { return 3 * k - 12; }

__device__ __forceinline__ uint32_t quantize(float x, float lo, float inv_extent, float cells, uint32_t qmax)
{
    const float q = (x - lo) * inv_extent * cells;
    // Origins outside the box (or NaN) clamp to its faces.
    if (!(q > 0.0f)) return 0u;
    return q >= (float)qmax ? qmax : (uint32_t)q;
}

// Bits 0..9 of x moved to bits 0, 3, 6, ..., 27 (the usual magic-number
// interleave), so three spread coordinates OR into a Morton code.
__device__ __forceinline__ uint32_t spread3(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
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
    const uint32_t m = spread3(qx) | (spread3(qy) << 1) | (spread3(qz) << 2);
    const uint32_t oct = (dd.x < 0.0f ? 1u : 0u) | (dd.y < 0.0f ? 2u : 0u) | (dd.z < 0.0f ? 4u : 0u);
    return (oct << (3 * k)) | m;
}

template <int P>
__device__ __forceinline__ uint32_t digit_of(uint32_t key, uint32_t k)
{
    if constexpr (P == kWhole) return key;
    else if constexpr (P == kLow) return key & ((1u << low_bits(k)) - 1u);
    else return key >> low_bits(k);
}

// Adds one to counter[digit] for every valid lane and returns a distinct
// previous value to each (the full warp calls this together; invalid lanes
// get an unused value).  Small histograms aggregate equal digits in the warp
// first: one lane per digit adds the group's size, and each lane takes the
// group's base plus its rank among the group's lanes, in lane order.
__device__ __forceinline__ uint32_t take(uint32_t* counter, uint32_t digit, bool valid, bool aggregate)
{
    if (!aggregate) return valid ? atomicAdd(&counter[digit], 1u) : 0u;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t tag = valid ? digit : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, tag);
    const unsigned leader = __ffs(peers) - 1u;
    uint32_t base = 0;
    if (valid && lane == leader) base = atomicAdd(&counter[digit], (uint32_t)__popc(peers));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

// Step 1: the tile's digits counted in shared memory, stored as row t of cnt.
// The first pass computes each ray's key from the ray and keeps it in keys.
template <int P>
__global__ void __launch_bounds__(kTileThreads, 2) k_tile_count(const rb2::ReorderArgs a, uint32_t nb)
{
    extern __shared__ uint32_t s_h[];
    const bool agg = nb <= kWarpAggMax;
    const uint32_t warp0 = (threadIdx.x & ~31u), lane = threadIdx.x & 31u;
    for (uint32_t t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) s_h[i] = 0u;
        __syncthreads();
        const rb2::ReorderTile tl = a.tiles[t];
        const uint64_t s0 = a.start[tl.job];
        // Whole warps step together (the aggregation needs every lane); two
        // entries per lane per step keep two loads in flight.
        for (uint32_t w = tl.begin + warp0; w < tl.end; w += 2 * kTileThreads) {
            const uint32_t s1 = w + lane, s2 = w + kTileThreads + lane;
            const bool v1 = s1 < tl.end, v2 = s2 < tl.end;
            uint32_t k1 = 0, k2 = 0;
            if constexpr (P == kHigh) {
                if (v1) k1 = a.pairs[s1].x;
                if (v2) k2 = a.pairs[s2].x;
            } else {
                if (v1) k1 = key_of(a, tl.job, s1 - s0);
                if (v2) k2 = key_of(a, tl.job, s2 - s0);
                if (v1) a.keys[s1] = k1;
                if (v2) a.keys[s2] = k2;
            }
            take(s_h, digit_of<P>(k1, a.bits), v1, agg);
            if (__any_sync(0xFFFFFFFFu, v2)) take(s_h, digit_of<P>(k2, a.bits), v2, agg);
        }
        __syncthreads();
        uint32_t* row = a.cnt + (uint64_t)t * nb;
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) row[i] = s_h[i];
        __syncthreads();
    }
}

// Step 2: per (job, bucket), an exclusive scan down the job's tiles, in place;
// the bucket's total goes to tot.
__global__ void k_tile_columns(const rb2::ReorderArgs a, uint32_t nb)
{
    constexpr uint32_t kRows = 8;  // rows loaded together, so their loads overlap
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
        a.tot[(uint64_t)j * nb + b] = run;
    }
}

// Step 4: the tile's first position in every bucket (bucket start + the
// tile's offset inside it) in shared memory; each entry takes the next one.
template <int P>
__global__ void __launch_bounds__(kTileThreads) k_tile_scatter(const rb2::ReorderArgs a, uint32_t nb)
{
    extern __shared__ uint32_t s_off[];
    const bool agg = nb <= kWarpAggMax;
    const uint32_t warp0 = (threadIdx.x & ~31u), lane = threadIdx.x & 31u;
    for (uint32_t t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
        const rb2::ReorderTile tl = a.tiles[t];
        const uint32_t* row = a.cnt + (uint64_t)t * nb;
        const uint32_t* base = a.tot + (uint64_t)tl.job * nb;
        for (uint32_t i = threadIdx.x; i < nb; i += kTileThreads) s_off[i] = base[i] + row[i];
        __syncthreads();
        for (uint32_t w = tl.begin + warp0; w < tl.end; w += kTileThreads) {
            const uint32_t s = w + lane;
            const bool v = s < tl.end;
            uint32_t key = 0, slot = s;
            if constexpr (P == kHigh) {
                if (v) {
                    const uint2 pr = a.pairs[s];
                    key = pr.x;
                    slot = pr.y;
                }
            } else {
                if (v) key = a.keys[s];
            }
            const uint32_t pos = take(s_off, digit_of<P>(key, a.bits), v, agg);
            if (v) {
                if constexpr (P == kLow) a.pairs[pos] = make_uint2(key, slot);
                else a.perm[pos] = slot;
            }
        }
        __syncthreads();
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
    const int smem = (int)(sizeof(uint32_t) << kReorderHighBits);
    cudaError_t e = cudaSuccess;
    const void* fns[] = {(const void*)k_tile_count<kWhole>, (const void*)k_tile_count<kLow>,
                         (const void*)k_tile_count<kHigh>, (const void*)k_tile_scatter<kWhole>,
                         (const void*)k_tile_scatter<kLow>, (const void*)k_tile_scatter<kHigh>};
    for (const void* f : fns)
        if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) break;
    return e;
}

namespace {

template <int P>
cudaError_t pass_enqueue(const ReorderArgs& a, uint32_t nb, cudaStream_t s)
{
    const size_t smem = sizeof(uint32_t) * nb;
    k_tile_count<P><<<a.n_tiles, kTileThreads, smem, s>>>(a, nb);
    const dim3 cols((nb + 255) / 256, std::min<uint32_t>(a.n_jobs, 65535u));
    k_tile_columns<<<cols, 256, 0, s>>>(a, nb);
    cudaError_t e = scan_enqueue(a.tot, (uint64_t)a.n_jobs * nb, a.chunk_sums, s);
    if (e != cudaSuccess) return e;
    k_tile_scatter<P><<<a.n_tiles, kTileThreads, smem, s>>>(a, nb);
    return cudaGetLastError();
}

}  // namespace

cudaError_t reorder_enqueue(const ReorderArgs& a, cudaStream_t s)
{
    if (a.total == 0 || a.n_tiles == 0) return cudaSuccess;
    if (a.bits <= kReorderOnePassMaxBits) return pass_enqueue<kWhole>(a, 1u << (3 + 3 * a.bits), s);
    cudaError_t e = pass_enqueue<kLow>(a, 1u << (3 * a.bits - 12), s);
    if (e != cudaSuccess) return e;
    return pass_enqueue<kHigh>(a, 1u << kReorderHighBits, s);
}

}  // namespace rb2
