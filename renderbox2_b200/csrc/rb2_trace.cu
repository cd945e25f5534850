// Tracer: device BVH upload and the persistent while-while traversal kernel
// for sm_100a, plus camera-ray generation.
//
// Traversal follows the reference's Aila-Laine persistent kernel
// (accelerators/sbvh/kepler_dynamic_fetch.h:67-363) and single-ray trace_ray
// (accelerators/sbvh/cuda_tracer_functions.cu:42-279): Compact2 nodes (64 B,
// two child boxes), Woop triangles (48 B) with a -0.0 terminator per leaf, a
// 64-entry stack, near child first, at most one postponed leaf, a warp vote
// that stops node traversal once every busy lane holds a leaf, and warps that
// refill from a global ray queue when fewer than `fetch_threshold` lanes are
// still busy.  B200 specifics: plain global loads through the non-coherent
// path (LDG.128) instead of texture objects, full-warp *_sync votes
// (independent thread scheduling), one queue counter per launch slot so
// traces on different streams do not share a counter, and a stack guard that
// records a status bit instead of writing out of bounds.
//
// Arithmetic is pinned: __fmaf_rn / __fmul_rn / __fdiv_rn in the exact order
// the CPU oracle uses, so hits, t, u and v are bit-identical to it.
#include "rb2.h"
#include "rb2_internal.h"
#include "rb2_render.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

namespace rb2 {
const HostBvh& host_of(const rb2_host_bvh* b);
}

namespace rb2dev {

constexpr int kSentinel = 0x76543210;
constexpr int kStackSize = 64;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlock = 128;
constexpr uint32_t kStatusStack = 1u;

enum Mode { kClosest = 0, kAny = 1, kOcclusion = 2 };

struct TraceArgs {
    const float4* __restrict__ nodes;
    const float4* __restrict__ woop;
    const uint32_t* __restrict__ triidx;
    const float4* __restrict__ rays;
    const uint8_t* __restrict__ mask;
    int4* __restrict__ hits;
    uint8_t* __restrict__ occl;
    unsigned int* counter;
    unsigned int* status;
    uint32_t n;
    uint32_t fetch_threshold;
};

__device__ __forceinline__ float fmin_s(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_s(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float imin_f(float a, float b) { return __int_as_float(min(__float_as_int(a), __float_as_int(b))); }
__device__ __forceinline__ float imax_f(float a, float b) { return __int_as_float(max(__float_as_int(a), __float_as_int(b))); }

__device__ __forceinline__ float span_begin(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imax_f(imax_f(fmin_s(a0, a1), fmin_s(b0, b1)), imax_f(imin_f(c0, c1), d));
}
__device__ __forceinline__ float span_end(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imin_f(imin_f(fmax_s(a0, a1), fmax_s(b0, b1)), imin_f(imax_f(c0, c1), d));
}

__device__ __forceinline__ float safe_rcp(float d)
{
    const float ooeps = 0x1p-80f;
    return __fdiv_rn(1.0f, fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

template <int MODE>
__device__ __forceinline__ void write_result(const TraceArgs& a, uint32_t ray, int hitIndex, float t, float u, float v)
{
    if (MODE == kOcclusion) {
        a.occl[ray] = hitIndex >= 0 ? 1 : 0;
    } else {
        int prim = hitIndex >= 0 ? (int)__ldg(a.triidx + hitIndex) : -1;
        a.hits[ray] = make_int4(prim, __float_as_int(t), __float_as_int(hitIndex >= 0 ? u : 0.0f),
                                __float_as_int(hitIndex >= 0 ? v : 0.0f));
    }
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, 8) k_trace(TraceArgs a)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;

    int stack[kStackSize + 2];
    int sp = 0;
    int nodeAddr = kSentinel, leafAddr = 0, hitIndex = -1;
    float ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0;
    float idx = 0, idy = 0, idz = 0, oodx = 0, oody = 0, oodz = 0;
    float tmin = 0, hitT = 0, hu = 0, hv = 0;
    uint32_t rayidx = 0;
    bool has_ray = false, retired = false;

    for (;;) {
        // ---- refill: lanes without a ray take the next indices from the queue.
        const bool need = !has_ray && !retired;
        const unsigned needm = __ballot_sync(kFull, need);
        if (needm) {
            const int leader = __ffs(needm) - 1;
            unsigned base = 0;
            if ((int)lane == leader) base = atomicAdd(a.counter, (unsigned)__popc(needm));
            base = __shfl_sync(kFull, base, leader);
            if (need) {
                rayidx = base + (unsigned)__popc(needm & lt_mask);
                if (rayidx >= a.n) {
                    retired = true;
                } else if (a.mask != nullptr && a.mask[rayidx] == 0) {
                    const float4 d4 = __ldg(a.rays + 2 * (size_t)rayidx + 1);
                    write_result<MODE>(a, rayidx, -1, d4.w, 0.0f, 0.0f);
                } else {
                    const float4 o4 = __ldg(a.rays + 2 * (size_t)rayidx + 0);
                    const float4 d4 = __ldg(a.rays + 2 * (size_t)rayidx + 1);
                    ox = o4.x; oy = o4.y; oz = o4.z; tmin = o4.w;
                    dx = d4.x; dy = d4.y; dz = d4.z; hitT = d4.w;
                    idx = safe_rcp(dx); idy = safe_rcp(dy); idz = safe_rcp(dz);
                    oodx = __fmul_rn(ox, idx); oody = __fmul_rn(oy, idy); oodz = __fmul_rn(oz, idz);
                    stack[0] = kSentinel;
                    sp = 0;
                    leafAddr = 0;
                    nodeAddr = 0;
                    hitIndex = -1;
                    hu = hv = 0.0f;
                    has_ray = true;
                }
            }
        }
        if (__all_sync(kFull, retired)) break;

        // ---- traversal until too few lanes are busy.
        while (__any_sync(kFull, has_ray)) {
            // Inner nodes until every busy lane has postponed a leaf.
            for (;;) {
                const bool in = has_ray && (unsigned)nodeAddr < (unsigned)kSentinel;
                if (!__any_sync(kFull, in)) break;
                if (in) {
                    const float4* np = a.nodes + nodeAddr;
                    const float4 n0xy = __ldg(np + 0);
                    const float4 n1xy = __ldg(np + 1);
                    const float4 nz = __ldg(np + 2);
                    const float4 cn = __ldg(np + 3);
                    int c0 = __float_as_int(cn.x), c1 = __float_as_int(cn.y);

                    const float c0lox = __fmaf_rn(n0xy.x, idx, -oodx);
                    const float c0hix = __fmaf_rn(n0xy.y, idx, -oodx);
                    const float c0loy = __fmaf_rn(n0xy.z, idy, -oody);
                    const float c0hiy = __fmaf_rn(n0xy.w, idy, -oody);
                    const float c0loz = __fmaf_rn(nz.x, idz, -oodz);
                    const float c0hiz = __fmaf_rn(nz.y, idz, -oodz);
                    const float c1loz = __fmaf_rn(nz.z, idz, -oodz);
                    const float c1hiz = __fmaf_rn(nz.w, idz, -oodz);
                    const float c0min = span_begin(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, tmin);
                    const float c0max = span_end(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, hitT);
                    const float c1lox = __fmaf_rn(n1xy.x, idx, -oodx);
                    const float c1hix = __fmaf_rn(n1xy.y, idx, -oodx);
                    const float c1loy = __fmaf_rn(n1xy.z, idy, -oody);
                    const float c1hiy = __fmaf_rn(n1xy.w, idy, -oody);
                    const float c1min = span_begin(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, tmin);
                    const float c1max = span_end(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, hitT);

                    const bool swp = c1min < c0min;
                    const bool t0 = c0max >= c0min;
                    const bool t1 = c1max >= c1min;
                    if (!t0 && !t1) {
                        nodeAddr = stack[sp--];
                    } else {
                        nodeAddr = t0 ? c0 : c1;
                        if (t0 && t1) {
                            if (swp) { const int tmp = nodeAddr; nodeAddr = c1; c1 = tmp; }
                            if (sp >= kStackSize) {
                                atomicOr(a.status, kStatusStack);
                                nodeAddr = kSentinel;  // abandon this ray; reported as a miss
                                leafAddr = 0;
                                hitIndex = -1;
                            } else {
                                stack[++sp] = c1;
                            }
                        }
                    }
                    if (nodeAddr < 0 && leafAddr >= 0) {
                        leafAddr = nodeAddr;
                        nodeAddr = stack[sp--];
                    }
                }
                if (!__any_sync(kFull, in && leafAddr >= 0)) break;
            }

            // Postponed leaves.
            if (has_ray) {
                while (leafAddr < 0) {
                    for (int triAddr = ~leafAddr;; triAddr += 3) {
                        const float4* wp = a.woop + triAddr;
                        const float4 v00 = __ldg(wp + 0);
                        const float4 v11 = __ldg(wp + 1);
                        const float4 v22 = __ldg(wp + 2);
                        if (__float_as_int(v00.x) == (int)0x80000000) break;

                        const float Oz = __fmaf_rn(-oz, v00.z, __fmaf_rn(-oy, v00.y, __fmaf_rn(-ox, v00.x, v00.w)));
                        const float Dz = __fmaf_rn(dz, v00.z, __fmaf_rn(dy, v00.y, __fmul_rn(dx, v00.x)));
                        const float t = __fmul_rn(Oz, __fdiv_rn(1.0f, Dz));
                        if (t > tmin && t < hitT) {
                            const float Ox = __fmaf_rn(oz, v11.z, __fmaf_rn(oy, v11.y, __fmaf_rn(ox, v11.x, v11.w)));
                            const float Dx = __fmaf_rn(dz, v11.z, __fmaf_rn(dy, v11.y, __fmul_rn(dx, v11.x)));
                            const float u = __fmaf_rn(t, Dx, Ox);
                            if (u >= 0.0f) {
                                const float Oy = __fmaf_rn(oz, v22.z, __fmaf_rn(oy, v22.y, __fmaf_rn(ox, v22.x, v22.w)));
                                const float Dy = __fmaf_rn(dz, v22.z, __fmaf_rn(dy, v22.y, __fmul_rn(dx, v22.x)));
                                const float v = __fmaf_rn(t, Dy, Oy);
                                if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                                    hitT = t;
                                    hu = u;
                                    hv = v;
                                    hitIndex = triAddr;
                                    if (MODE != kClosest) {
                                        nodeAddr = kSentinel;
                                        break;
                                    }
                                }
                            }
                        }
                    }
                    leafAddr = nodeAddr;
                    if (nodeAddr < 0) nodeAddr = stack[sp--];
                }
                if (nodeAddr == kSentinel) {
                    write_result<MODE>(a, rayidx, hitIndex, hitT, hu, hv);
                    has_ray = false;
                }
            }
            // Dynamic fetch (kepler_dynamic_fetch.h:308-310).
            if ((unsigned)__popc(__ballot_sync(kFull, has_ray)) < a.fetch_threshold) break;
        }
    }
}

// ---- camera rays ------------------------------------------------------------------
struct CamArgs {
    float r2c[16];
    float c2w[16];
    uint32_t width, height, spp, jitter;
    uint64_t seed;
};

// Row-vector products evaluated left to right without contraction, like the
// reference's float4 dot (helper_math) on Matrix4x4 rows (core/transform.h:186-199).
__device__ __forceinline__ float row_dot(const float* r, float x, float y, float z, float w)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r[0], x), __fmul_rn(r[1], y)), __fmul_rn(r[2], z)), __fmul_rn(r[3], w));
}

__device__ __forceinline__ void camera_ray(const float* r2c, const float* c2w, float x, float y, float4& o4, float4& d4)
{
    // p_camera = raster_to_camera(point (x, y, 0)), divided by w.
    float px = row_dot(r2c + 0, x, y, 0.0f, 1.0f);
    float py = row_dot(r2c + 4, x, y, 0.0f, 1.0f);
    float pz = row_dot(r2c + 8, x, y, 0.0f, 1.0f);
    float pw = row_dot(r2c + 12, x, y, 0.0f, 1.0f);
    px = __fdiv_rn(px, pw); py = __fdiv_rn(py, pw); pz = __fdiv_rn(pz, pw);
    // normalize = v * (1 / sqrt(dot(v, v)))
    float dd = __fadd_rn(__fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py)), __fmul_rn(pz, pz));
    float inv = __fdiv_rn(1.0f, __fsqrt_rn(dd));
    float dxc = __fmul_rn(px, inv), dyc = __fmul_rn(py, inv), dzc = __fmul_rn(pz, inv);
    // camera_to_world: origin as a point, direction as a vector.
    float oxw = row_dot(c2w + 0, 0.0f, 0.0f, 0.0f, 1.0f);
    float oyw = row_dot(c2w + 4, 0.0f, 0.0f, 0.0f, 1.0f);
    float ozw = row_dot(c2w + 8, 0.0f, 0.0f, 0.0f, 1.0f);
    float oww = row_dot(c2w + 12, 0.0f, 0.0f, 0.0f, 1.0f);
    o4 = make_float4(__fdiv_rn(oxw, oww), __fdiv_rn(oyw, oww), __fdiv_rn(ozw, oww), 0.0f);
    d4 = make_float4(row_dot(c2w + 0, dxc, dyc, dzc, 0.0f), row_dot(c2w + 4, dxc, dyc, dzc, 0.0f),
                     row_dot(c2w + 8, dxc, dyc, dzc, 0.0f), 3.402823466e+38f);
}

__device__ __forceinline__ uint32_t pcg_hash(uint64_t v)
{
    // One PCG32 output step applied to a counter (O'Neill 2014 output function).
    uint64_t state = v * 6364136223846793005ULL + 1442695040888963407ULL;
    uint32_t xs = (uint32_t)(((state >> 18u) ^ state) >> 27u);
    uint32_t rot = (uint32_t)(state >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}

__global__ void k_camera_rays(CamArgs c, float4* rays)
{
    const uint64_t total = (uint64_t)c.width * c.height * c.spp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pix = i / c.spp;
        const uint32_t px = (uint32_t)(pix % c.width), py = (uint32_t)(pix / c.width);
        float jx = 0.5f, jy = 0.5f;
        if (c.jitter) {
            uint64_t key = (c.seed * 0x9E3779B97F4A7C15ULL) ^ (i * 2ULL);
            jx = (float)(pcg_hash(key) >> 8) * (1.0f / 16777216.0f);
            jy = (float)(pcg_hash(key + 1) >> 8) * (1.0f / 16777216.0f);
        }
        float4 o, d;
        camera_ray(c.r2c, c.c2w, (float)px + jx, (float)py + jy, o, d);
        rays[2 * i + 0] = o;
        rays[2 * i + 1] = d;
    }
}

__global__ void k_camera_rays_at(CamArgs c, const float2* xy, uint32_t n, float4* rays)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 o, d;
        const float2 p = xy[i];
        camera_ray(c.r2c, c.c2w, p.x, p.y, o, d);
        rays[2 * (size_t)i + 0] = o;
        rays[2 * (size_t)i + 1] = d;
    }
}

}  // namespace rb2dev

// ======================================================================= host side
using namespace rb2;

struct rb2_tracer {
    int device = 0;
    int num_sms = 0;
    float4* d_nodes = nullptr;
    float4* d_woop = nullptr;
    uint32_t* d_triidx = nullptr;
    uint64_t n_nodes_u4 = 0, n_woop_u4 = 0;
    unsigned int* d_words = nullptr;  // [0, kSlots) queue heads, [kSlots] status
    uint32_t slot = 0;
    rb2_launch_config cfg{};
    int occ[3] = {0, 0, 0};
    // scratch for the host-buffer path
    float4* d_rays = nullptr;
    int4* d_hits = nullptr;
    uint8_t* d_mask = nullptr;
    uint64_t scratch_cap = 0;
    uint64_t device_bytes = 0;
    std::mutex mu;
};

namespace {

constexpr uint32_t kSlots = 256;

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(RB2_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RB2_CUDA(call, what)                         \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

template <int MODE>
int launch_trace(rb2_tracer* t, const float* d_rays, uint32_t n, const uint8_t* d_mask, int4* d_hits, uint8_t* d_occ,
                 cudaStream_t s)
{
    if (n == 0) return RB2_OK;
    uint32_t slot;
    {
        std::lock_guard<std::mutex> g(t->mu);
        slot = t->slot++ % kSlots;
    }
    RB2_CUDA(cudaMemsetAsync(t->d_words + slot, 0, sizeof(unsigned int), s), "queue reset");
    rb2dev::TraceArgs a;
    a.nodes = t->d_nodes;
    a.woop = t->d_woop;
    a.triidx = t->d_triidx;
    a.rays = reinterpret_cast<const float4*>(d_rays);
    a.mask = d_mask;
    a.hits = d_hits;
    a.occl = d_occ;
    a.counter = t->d_words + slot;
    a.status = t->d_words + kSlots;
    a.n = n;
    a.fetch_threshold = t->cfg.fetch_threshold ? t->cfg.fetch_threshold : 20u;
    int per_sm = t->cfg.ctas_per_sm ? (int)t->cfg.ctas_per_sm : t->occ[MODE];
    uint64_t warps_needed = ((uint64_t)n + 31) / 32;
    uint64_t blocks = (uint64_t)t->num_sms * (uint64_t)std::max(1, per_sm);
    blocks = std::min<uint64_t>(blocks, (warps_needed + rb2dev::kBlock / 32 - 1) / (rb2dev::kBlock / 32));
    blocks = std::max<uint64_t>(blocks, 1);
    rb2dev::k_trace<MODE><<<(unsigned)blocks, rb2dev::kBlock, 0, s>>>(a);
    RB2_CUDA(cudaGetLastError(), "trace launch");
    return RB2_OK;
}

}  // namespace

extern "C" {

int rb2_tracer_create(const rb2_host_bvh* bvh, rb2_tracer** out)
{
    if (!bvh || !out) return fail(RB2_EINVAL, "null argument");
    *out = nullptr;
    const HostBvh& h = host_of(bvh);
    uint32_t depth = 0;
    int rc = validate_compact2(h.nodes.data(), h.nodes.size() / 4, h.woop.data(), h.woop.size() / 4, h.triidx.data(),
                               h.triidx.size(), 0, &depth);
    if (rc) return rc;
    std::unique_ptr<rb2_tracer> t(new rb2_tracer());
    RB2_CUDA(cudaGetDevice(&t->device), "cudaGetDevice");
    RB2_CUDA(cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, t->device), "SM count");
    t->n_nodes_u4 = h.nodes.size() / 4;
    t->n_woop_u4 = h.woop.size() / 4;
    // Two spare uint4 after the Woop buffer: the kernel fetches a triangle's
    // three rows before testing the first for the terminator.
    const size_t nb = h.nodes.size() * 4, wb = (h.woop.size() + 8) * 4, ib = h.triidx.size() * 4 + 16;
    auto cleanup = [&]() {
        cudaFree(t->d_nodes); cudaFree(t->d_woop); cudaFree(t->d_triidx); cudaFree(t->d_words);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&t->d_nodes, nb)) != cudaSuccess || (e = cudaMalloc(&t->d_woop, wb)) != cudaSuccess ||
        (e = cudaMalloc(&t->d_triidx, ib)) != cudaSuccess ||
        (e = cudaMalloc(&t->d_words, (kSlots + 1) * sizeof(unsigned int))) != cudaSuccess) {
        cleanup();
        return fail(RB2_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpy(t->d_nodes, h.nodes.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_woop, 0, wb)) != cudaSuccess ||
        (e = cudaMemcpy(t->d_woop, h.woop.data(), h.woop.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_triidx, 0, ib)) != cudaSuccess ||
        (e = cudaMemcpy(t->d_triidx, h.triidx.data(), h.triidx.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_words, 0, (kSlots + 1) * sizeof(unsigned int))) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "BVH upload");
    }
    t->device_bytes = nb + wb + ib + (kSlots + 1) * sizeof(unsigned int);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&t->occ[0], rb2dev::k_trace<0>, rb2dev::kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&t->occ[1], rb2dev::k_trace<1>, rb2dev::kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&t->occ[2], rb2dev::k_trace<2>, rb2dev::kBlock, 0);
    *out = t.release();
    return RB2_OK;
}

int rb2_tracer_destroy(rb2_tracer* t)
{
    if (!t) return RB2_OK;
    cudaFree(t->d_nodes);
    cudaFree(t->d_woop);
    cudaFree(t->d_triidx);
    cudaFree(t->d_words);
    cudaFree(t->d_rays);
    cudaFree(t->d_hits);
    cudaFree(t->d_mask);
    delete t;
    return RB2_OK;
}

int rb2_tracer_set_launch(rb2_tracer* t, const rb2_launch_config* cfg)
{
    if (!t || !cfg) return fail(RB2_EINVAL, "null argument");
    if (cfg->block_threads && cfg->block_threads != (uint32_t)rb2dev::kBlock)
        return fail(RB2_ENOTSUP, "the traversal kernel is compiled for 128-thread CTAs");
    if (cfg->fetch_threshold > 32) return fail(RB2_EINVAL, "fetch_threshold must be <= 32");
    t->cfg = *cfg;
    return RB2_OK;
}

int rb2_tracer_device_bytes(const rb2_tracer* t, uint64_t* bytes)
{
    if (!t || !bytes) return fail(RB2_EINVAL, "null argument");
    *bytes = t->device_bytes;
    return RB2_OK;
}

int rb2_trace(rb2_tracer* t, const float* d_rays, uint32_t n, int any_hit, const uint8_t* d_mask, rb2_hit* d_hits,
              void* stream)
{
    if (!t || (n && (!d_rays || !d_hits))) return fail(RB2_EINVAL, "null argument");
    if (((uintptr_t)d_rays | (uintptr_t)d_hits) & 15u) return fail(RB2_EINVAL, "rays and hits must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    int4* hits = reinterpret_cast<int4*>(d_hits);
    return any_hit ? launch_trace<rb2dev::kAny>(t, d_rays, n, d_mask, hits, nullptr, s)
                   : launch_trace<rb2dev::kClosest>(t, d_rays, n, d_mask, hits, nullptr, s);
}

int rb2_trace_occlusion(rb2_tracer* t, const float* d_rays, uint32_t n, const uint8_t* d_mask, uint8_t* d_occluded,
                        void* stream)
{
    if (!t || (n && (!d_rays || !d_occluded))) return fail(RB2_EINVAL, "null argument");
    if ((uintptr_t)d_rays & 15u) return fail(RB2_EINVAL, "rays must be 16-byte aligned");
    return launch_trace<rb2dev::kOcclusion>(t, d_rays, n, d_mask, nullptr, d_occluded, (cudaStream_t)stream);
}

int rb2_trace_host(rb2_tracer* t, const float* h_rays, uint32_t n, int any_hit, const uint8_t* h_mask, rb2_hit* h_hits,
                   void* stream)
{
    if (!t || (n && (!h_rays || !h_hits))) return fail(RB2_EINVAL, "null argument");
    if (n == 0) return RB2_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (n > t->scratch_cap) {
        RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
        cudaFree(t->d_rays); cudaFree(t->d_hits); cudaFree(t->d_mask);
        t->d_rays = nullptr; t->d_hits = nullptr; t->d_mask = nullptr;
        t->scratch_cap = 0;
        cudaError_t e;
        if ((e = cudaMalloc(&t->d_rays, (size_t)n * 32)) != cudaSuccess || (e = cudaMalloc(&t->d_hits, (size_t)n * 16)) != cudaSuccess ||
            (e = cudaMalloc(&t->d_mask, (size_t)n)) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("scratch allocation: ") + cudaGetErrorString(e));
        t->scratch_cap = n;
    }
    RB2_CUDA(cudaMemcpyAsync(t->d_rays, h_rays, (size_t)n * 32, cudaMemcpyHostToDevice, s), "ray upload");
    if (h_mask) RB2_CUDA(cudaMemcpyAsync(t->d_mask, h_mask, n, cudaMemcpyHostToDevice, s), "mask upload");
    int rc = rb2_trace(t, reinterpret_cast<const float*>(t->d_rays), n, any_hit, h_mask ? t->d_mask : nullptr,
                       reinterpret_cast<rb2_hit*>(t->d_hits), stream);
    if (rc) return rc;
    RB2_CUDA(cudaMemcpyAsync(h_hits, t->d_hits, (size_t)n * 16, cudaMemcpyDeviceToHost, s), "hit download");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    return RB2_OK;
}

int rb2_tracer_status(rb2_tracer* t, uint32_t* status, void* stream)
{
    if (!t || !status) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    RB2_CUDA(cudaMemcpyAsync(status, t->d_words + kSlots, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "status read");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    return RB2_OK;
}

int rb2_camera_rays(const rb2_camera* cam, uint32_t spp, uint64_t seed, int jitter, float* d_rays, void* stream)
{
    if (!cam || !d_rays || spp == 0) return fail(RB2_EINVAL, "bad camera-ray arguments");
    rb2dev::CamArgs c;
    std::memcpy(c.r2c, cam->raster_to_camera, sizeof(c.r2c));
    std::memcpy(c.c2w, cam->camera_to_world, sizeof(c.c2w));
    c.width = cam->width; c.height = cam->height; c.spp = spp; c.jitter = jitter ? 1u : 0u; c.seed = seed;
    uint64_t total = (uint64_t)cam->width * cam->height * spp;
    unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
    rb2dev::k_camera_rays<<<std::max(1u, blocks), 256, 0, (cudaStream_t)stream>>>(c, reinterpret_cast<float4*>(d_rays));
    RB2_CUDA(cudaGetLastError(), "camera launch");
    return RB2_OK;
}

int rb2_camera_rays_at(const rb2_camera* cam, const float* d_raster_xy, uint32_t n, float* d_rays, void* stream)
{
    if (!cam || (n && (!d_raster_xy || !d_rays))) return fail(RB2_EINVAL, "bad camera-ray arguments");
    if (n == 0) return RB2_OK;
    rb2dev::CamArgs c;
    std::memcpy(c.r2c, cam->raster_to_camera, sizeof(c.r2c));
    std::memcpy(c.c2w, cam->camera_to_world, sizeof(c.c2w));
    c.width = cam->width; c.height = cam->height; c.spp = 1; c.jitter = 0; c.seed = 0;
    unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    rb2dev::k_camera_rays_at<<<std::max(1u, blocks), 256, 0, (cudaStream_t)stream>>>(
        c, reinterpret_cast<const float2*>(d_raster_xy), n, reinterpret_cast<float4*>(d_rays));
    RB2_CUDA(cudaGetLastError(), "camera launch");
    return RB2_OK;
}

}  // extern "C"
