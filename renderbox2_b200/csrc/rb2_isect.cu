// Intersection records (rb2_trace_isect), the bulk entry of the header-only
// device traversal (rb2_trace_per_thread) and the device view of a scene.
//
// rb2_trace_isect runs the persistent while-while traversal with a ray source
// whose finish() writes the reference's SoA intersection record directly
// (accelerators/sbvh/kepler_dynamic_fetch.h:313-355), so hit records never
// make a round trip through HBM before the record is built.
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_device.cuh"
#include "rb2_internal.h"
#include "rb2_render.h"
#include "rb2_render_internal.h"
#include "rb2_traverse.cuh"
#include "rb2_traverse_cw8.cuh"

#include <cuda_runtime.h>

#include <algorithm>

namespace rb2dev {

struct IsectSource {
    const float4* nodes;
    const float4* woop;
    const uint32_t* triidx;
    const float4* rays;
    const uint8_t* mask;
    uint64_t n;
    uint32_t mode;
    unsigned long long* head;
    rb2_isect_buffer out;
    rb2_dev_scene scene;

    __device__ __forceinline__ void claim(unsigned count, unsigned long long& b1, unsigned& n1, unsigned long long& b2)
    {
        b1 = atomicAdd(head, (unsigned long long)count);
        n1 = count;
        b2 = 0;
    }

    __device__ __forceinline__ int fetch(unsigned long long slot, Lane& L) const
    {
        if (slot >= n) return 0;
        if (mask != nullptr && mask[slot] == 0) {
            if (out.intersected) out.intersected[slot] = 0;
            return -1;
        }
        L.nodes = nodes;
        L.woop = woop;
        L.set_tag(mode, 0);
        L.ray = (uint32_t)slot;
        setup_ray(L, __ldg(rays + 2 * slot), __ldg(rays + 2 * slot + 1));
        return 1;
    }

    __device__ __forceinline__ void finish(const Lane& L) const
    {
        const uint64_t r = L.ray;
        const bool hit = L.hitIndex >= 0;
        if (out.intersected) out.intersected[r] = hit ? 1 : 0;
        if (!hit || mode != kClosest) return;
        rb2_hit h;
        h.prim = (int32_t)__ldg(triidx + L.hitIndex);
        h.t = L.hitT;
        const float2 uv = hit_uv(L);
        h.u = uv.x;
        h.v = uv.y;
        rb2::Intersection is;
        rb2::fill_intersection(make_float4(L.ox, L.oy, L.oz, L.tmin), make_float4(L.dx, L.dy, L.dz, 0.0f), h, scene,
                               &is);
        if (out.position[0]) { out.position[0][r] = is.position.x; out.position[1][r] = is.position.y; out.position[2][r] = is.position.z; }
        if (out.geometric_normal[0]) { out.geometric_normal[0][r] = is.Ng.x; out.geometric_normal[1][r] = is.Ng.y; out.geometric_normal[2][r] = is.Ng.z; }
        if (out.shading_normal[0]) { out.shading_normal[0][r] = is.Ns.x; out.shading_normal[1][r] = is.Ns.y; out.shading_normal[2][r] = is.Ns.z; }
        if (out.incoming_direction[0]) { out.incoming_direction[0][r] = is.wi.x; out.incoming_direction[1][r] = is.wi.y; out.incoming_direction[2][r] = is.wi.z; }
        if (out.uv) reinterpret_cast<float2*>(out.uv)[r] = is.uv;
        if (out.primitive_id) out.primitive_id[r] = is.primitive_id;
        if (out.primitive_material_id) out.primitive_material_id[r] = is.primitive_material_id;
        if (out.front) out.front[r] = is.front;
        if (out.epsilon) out.epsilon[r] = is.epsilon;
    }
};

// LAYOUT: binary Compact2 or compressed 8-wide nodes (the tracer's layout).
template <int BLOCK, int LAYOUT>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
    k_trace_isect(const __grid_constant__ IsectSource src, uint32_t fetch_threshold, uint32_t node_threshold,
                  unsigned int* status)
{
    IsectSource s = src;
    if constexpr (LAYOUT == kLayoutCw8) persistent_trace_cw8(s, fetch_threshold, node_threshold, status);
    else persistent_trace(s, fetch_threshold, node_threshold, status);
}

__global__ void k_trace_per_thread(rb2_dev_bvh bvh, const float4* rays, const uint8_t* mask, uint32_t n, int any_hit,
                                   rb2_hit* out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldg(rays + 2 * (size_t)i), d = __ldg(rays + 2 * (size_t)i + 1);
    if (mask != nullptr && mask[i] == 0) {
        out[i] = rb2_hit{-1, d.w, 0.0f, 0.0f};
        return;
    }
    rb2_hit h;
    rb2::trace_ray(o, d, any_hit != 0, bvh, &h);
    out[i] = h;
}

}  // namespace rb2dev

using namespace rb2;

namespace {

int cuda_fail(cudaError_t e, const char* what) { return fail(rb2::cuda_status(e), std::string(what) + ": " + cudaGetErrorString(e)); }

#define RB2_CUDA(call, what)                               \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

bool misaligned(const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) != 0; }

}  // namespace

extern "C" {

int rb2_scene_dev_view(const rb2_scene_dev* s, rb2_dev_scene* out)
{
    if (!s || !out) return fail(RB2_EINVAL, "null argument");
    out->verts = s->d_verts;
    out->tris = s->d_tris;
    out->nv = s->nv;
    out->ntri = s->ntri;
    return RB2_OK;
}

int rb2_trace_isect(rb2_tracer* t, const rb2_scene_dev* scene, const float* d_rays, uint32_t n, int any_hit,
                    const uint8_t* d_mask, const rb2_isect_buffer* out, void* stream)
{
    rb2::Range nvtx_range("rb2_trace_isect");
    if (!t || !scene || !out || (n && !d_rays)) return fail(RB2_EINVAL, "null argument");
    if (misaligned(d_rays, 16)) return fail(RB2_EINVAL, "rays must be 16-byte aligned");
    if (out->uv && misaligned(out->uv, 8)) return fail(RB2_EINVAL, "uv must be 8-byte aligned");
    for (int k = 1; k < 3; k++) {
        if ((out->position[k] == nullptr) != (out->position[0] == nullptr) ||
            (out->geometric_normal[k] == nullptr) != (out->geometric_normal[0] == nullptr) ||
            (out->shading_normal[k] == nullptr) != (out->shading_normal[0] == nullptr) ||
            (out->incoming_direction[k] == nullptr) != (out->incoming_direction[0] == nullptr))
            return fail(RB2_EINVAL, "vector fields need all three planes or none");
    }
    if (n == 0) return RB2_OK;
    const cudaStream_t s = (cudaStream_t)stream;
    const DeviceBvhView bv = device_bvh(t, true);  // the compressed layout when the tracer uses it
    rb2dev::IsectSource src{};
    src.nodes = static_cast<const float4*>(bv.nodes);
    src.woop = static_cast<const float4*>(bv.woop);
    src.triidx = bv.triidx;
    src.rays = reinterpret_cast<const float4*>(d_rays);
    src.mask = d_mask;
    src.n = n;
    src.mode = any_hit ? rb2dev::kAny : rb2dev::kClosest;
    src.head = tracer_queue_counter(t);
    src.out = *out;
    int rc = rb2_scene_dev_view(scene, &src.scene);
    if (rc) return rc;
    RB2_CUDA(cudaMemsetAsync(src.head, 0, sizeof(unsigned long long), s), "queue reset");
    int dev = 0, sms = 0, per_sm = 0;
    RB2_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    RB2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    auto kern = bv.cw8 ? rb2dev::k_trace_isect<128, rb2dev::kLayoutCw8> : rb2dev::k_trace_isect<128, rb2dev::kLayoutBinary>;
    RB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0), "occupancy");
    uint64_t blocks = (uint64_t)sms * (uint64_t)std::max(1, per_sm);
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, ((uint64_t)n + 127) / 128));
    kern<<<(unsigned)blocks, 128, 0, s>>>(
        src, 20u, rb2dev::default_node_threshold(bv.cw8 ? rb2dev::kLayoutCw8 : rb2dev::kLayoutBinary), bv.status);
    RB2_CUDA(cudaGetLastError(), "isect launch");
    return RB2_OK;
}

int rb2_trace_per_thread(rb2_tracer* t, const float* d_rays, uint32_t n, int any_hit, const uint8_t* d_mask,
                         rb2_hit* d_hits, void* stream)
{
    if (!t || (n && (!d_rays || !d_hits))) return fail(RB2_EINVAL, "null argument");
    if (misaligned(d_rays, 16) || misaligned(d_hits, 16)) return fail(RB2_EINVAL, "rays and hits must be 16-byte aligned");
    if (n == 0) return RB2_OK;
    rb2_dev_bvh bvh;
    int rc = rb2_tracer_dev_bvh(t, &bvh);
    if (rc) return rc;
    const unsigned blocks = (unsigned)(((uint64_t)n + 127) / 128);
    rb2dev::k_trace_per_thread<<<blocks, 128, 0, (cudaStream_t)stream>>>(bvh, reinterpret_cast<const float4*>(d_rays),
                                                                          d_mask, n, any_hit, d_hits);
    RB2_CUDA(cudaGetLastError(), "per-thread trace launch");
    return RB2_OK;
}

}  // extern "C"
