/*
 * rb2_device.cuh -- header-only device traversal for CUDA kernels that trace
 * rays inside their own code (one thread per ray).
 *
 * Counterpart of the reference's __device__ trace_ray(const Ray&, bool anyhit,
 * Intersection*, nodes, tris, triIndices, SceneBuffer)
 * (accelerators/sbvh/cudatracerkernels.h:132-141, body
 * accelerators/sbvh/cuda_tracer_functions.cu:42-279).  Texture objects are
 * replaced by the plain 16-byte-aligned pointers of rb2_dev_bvh
 * (rb2_tracer_dev_bvh), the SceneBuffer by rb2_dev_scene
 * (rb2_scene_dev_view).
 *
 * Arithmetic: IEEE single precision, pinned operation by operation
 *   ray setup  idir = 1 / (|d| > 2^-80 ? d : copysign(2^-80, d)), ood = o * idir
 *   slab       fma(bound, idir, -ood); spans via signed-integer min/max of
 *              the float bit patterns (cudatracerkernels.h:213-256)
 *   Woop test  cuda_tracer_functions.cu:188-208 as FMA chains, t = Oz * (1/Dz)
 * Traversal order is the single-lane while-while loop: a leaf is tested as
 * soon as it is found (two when both children are leaves), so the result
 * (prim, t, u, v) does not depend on the other threads of the warp.  The
 * intersection record (rb2::Intersection) follows
 * accelerators/sbvh/kepler_dynamic_fetch.h:313-355 with no FMA contraction:
 * Ng = normalize(cross(v1 - v0, v2 - v0)), normalize(x) = x * (1/sqrt(dot)),
 * Ns = Ng, position = o + d t, wi = -d, front = dot(Ng, d) < 0,
 * uv of the accepted triangle, epsilon = 1e-3 t.
 *
 * The BVH must have been validated (every tracer's is): the 64-entry stack
 * cannot overflow for trees of depth <= 64; deeper input is rejected at
 * tracer creation, so no bound check is needed here.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb2.h"
#include "rb2_render.h"

namespace rb2 {

struct Intersection {
    float3 position;
    float3 Ng;
    float3 Ns;
    float3 wi;
    float2 uv;
    uint32_t primitive_id;
    uint32_t primitive_material_id;
    uint8_t front;
    uint8_t intersected;
    float epsilon;
};

namespace detail {

constexpr int kEntrySentinel = 0x76543210;

__device__ __forceinline__ float fmin_s(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_s(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float imin_f(float a, float b) { return __int_as_float(min(__float_as_int(a), __float_as_int(b))); }
__device__ __forceinline__ float imax_f(float a, float b) { return __int_as_float(max(__float_as_int(a), __float_as_int(b))); }
__device__ __forceinline__ float rcp_safe(float d)
{
    return __fdiv_rn(1.0f, fabsf(d) > 0x1p-80f ? d : copysignf(0x1p-80f, d));
}

}  // namespace detail

// Closest hit (any_hit == false) or the first accepted hit (any_hit == true)
// of the ray (o, tmin) + (d, tmax).  Returns true on a hit and fills `hit`
// (prim = original triangle id, t, u, v); on a miss hit = {-1, tmax, 0, 0}.
__device__ inline bool trace_ray(float4 o_tmin, float4 d_tmax, bool any_hit, const rb2_dev_bvh& bvh, rb2_hit* hit)
{
    using namespace detail;
    const float4* nodes = static_cast<const float4*>(bvh.nodes);
    const float4* woop = static_cast<const float4*>(bvh.woop);
    const float ox = o_tmin.x, oy = o_tmin.y, oz = o_tmin.z, tmin = o_tmin.w;
    const float dx = d_tmax.x, dy = d_tmax.y, dz = d_tmax.z;
    const float idx = rcp_safe(dx), idy = rcp_safe(dy), idz = rcp_safe(dz);
    const float oodx = __fmul_rn(ox, idx), oody = __fmul_rn(oy, idy), oodz = __fmul_rn(oz, idz);
    float hitT = d_tmax.w, hu = 0.0f, hv = 0.0f;
    int stack[66];
    int sp = 0;
    stack[0] = kEntrySentinel;
    int leafAddr = 0, nodeAddr = 0, hitIndex = -1;

    while (nodeAddr != kEntrySentinel) {
        while ((unsigned)nodeAddr < (unsigned)kEntrySentinel) {
            const float4* np = nodes + nodeAddr;
            const float4 a = __ldg(np + 0), b = __ldg(np + 1), z = __ldg(np + 2), c = __ldg(np + 3);
            int c0 = __float_as_int(c.x), c1 = __float_as_int(c.y);
            const float c0lox = __fmaf_rn(a.x, idx, -oodx), c0hix = __fmaf_rn(a.y, idx, -oodx);
            const float c0loy = __fmaf_rn(a.z, idy, -oody), c0hiy = __fmaf_rn(a.w, idy, -oody);
            const float c0loz = __fmaf_rn(z.x, idz, -oodz), c0hiz = __fmaf_rn(z.y, idz, -oodz);
            const float c1loz = __fmaf_rn(z.z, idz, -oodz), c1hiz = __fmaf_rn(z.w, idz, -oodz);
            const float c1lox = __fmaf_rn(b.x, idx, -oodx), c1hix = __fmaf_rn(b.y, idx, -oodx);
            const float c1loy = __fmaf_rn(b.z, idy, -oody), c1hiy = __fmaf_rn(b.w, idy, -oody);
            const float c0min = imax_f(imax_f(fmin_s(c0lox, c0hix), fmin_s(c0loy, c0hiy)), imax_f(imin_f(c0loz, c0hiz), tmin));
            const float c0max = imin_f(imin_f(fmax_s(c0lox, c0hix), fmax_s(c0loy, c0hiy)), imin_f(imax_f(c0loz, c0hiz), hitT));
            const float c1min = imax_f(imax_f(fmin_s(c1lox, c1hix), fmin_s(c1loy, c1hiy)), imax_f(imin_f(c1loz, c1hiz), tmin));
            const float c1max = imin_f(imin_f(fmax_s(c1lox, c1hix), fmax_s(c1loy, c1hiy)), imin_f(imax_f(c1loz, c1hiz), hitT));
            const bool t0 = c0max >= c0min, t1 = c1max >= c1min;
            if (!t0 && !t1) {
                nodeAddr = stack[sp--];
            } else {
                nodeAddr = t0 ? c0 : c1;
                if (t0 && t1) {
                    if (c1min < c0min) { const int tmp = nodeAddr; nodeAddr = c1; c1 = tmp; }
                    stack[++sp] = c1;
                }
            }
            if (nodeAddr < 0 && leafAddr >= 0) {
                leafAddr = nodeAddr;
                nodeAddr = stack[sp--];
            }
            if (leafAddr < 0) break;
        }
        while (leafAddr < 0) {
            for (int triAddr = ~leafAddr;; triAddr += 3) {
                const float4 w0 = __ldg(woop + triAddr);
                if (__float_as_int(w0.x) == (int)0x80000000) break;
                const float4 w1 = __ldg(woop + triAddr + 1), w2 = __ldg(woop + triAddr + 2);
                const float Oz = __fmaf_rn(-oz, w0.z, __fmaf_rn(-oy, w0.y, __fmaf_rn(-ox, w0.x, w0.w)));
                const float Dz = __fmaf_rn(dz, w0.z, __fmaf_rn(dy, w0.y, __fmul_rn(dx, w0.x)));
                const float t = __fmul_rn(Oz, __fdiv_rn(1.0f, Dz));
                if (t > tmin && t < hitT) {
                    const float Ox = __fmaf_rn(oz, w1.z, __fmaf_rn(oy, w1.y, __fmaf_rn(ox, w1.x, w1.w)));
                    const float Dx = __fmaf_rn(dz, w1.z, __fmaf_rn(dy, w1.y, __fmul_rn(dx, w1.x)));
                    const float u = __fmaf_rn(t, Dx, Ox);
                    if (u >= 0.0f) {
                        const float Oy = __fmaf_rn(oz, w2.z, __fmaf_rn(oy, w2.y, __fmaf_rn(ox, w2.x, w2.w)));
                        const float Dy = __fmaf_rn(dz, w2.z, __fmaf_rn(dy, w2.y, __fmul_rn(dx, w2.x)));
                        const float v = __fmaf_rn(t, Dy, Oy);
                        if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                            hitT = t; hu = u; hv = v; hitIndex = triAddr;
                            if (any_hit) { nodeAddr = kEntrySentinel; break; }
                        }
                    }
                }
            }
            leafAddr = nodeAddr;
            if (nodeAddr < 0) nodeAddr = stack[sp--];
        }
    }
    if (hitIndex >= 0) {
        hit->prim = (int32_t)__ldg(bvh.triidx + hitIndex);
        hit->t = hitT; hit->u = hu; hit->v = hv;
        return true;
    }
    hit->prim = -1; hit->t = d_tmax.w; hit->u = 0.0f; hit->v = 0.0f;
    return false;
}

// Intersection record of a closest hit `h` of ray (o, d) on `scene`.
__device__ inline void fill_intersection(float4 o, float4 d, const rb2_hit& h, const rb2_dev_scene& scene,
                                         Intersection* is)
{
    const float4* verts = static_cast<const float4*>(scene.verts);
    const uint4 tri = __ldg(static_cast<const uint4*>(scene.tris) + h.prim);
    const float4 a = __ldg(verts + tri.x), b = __ldg(verts + tri.y), c = __ldg(verts + tri.z);
    const float e1x = __fsub_rn(b.x, a.x), e1y = __fsub_rn(b.y, a.y), e1z = __fsub_rn(b.z, a.z);
    const float e2x = __fsub_rn(c.x, a.x), e2y = __fsub_rn(c.y, a.y), e2z = __fsub_rn(c.z, a.z);
    const float cx = __fsub_rn(__fmul_rn(e1y, e2z), __fmul_rn(e1z, e2y));
    const float cy = __fsub_rn(__fmul_rn(e1z, e2x), __fmul_rn(e1x, e2z));
    const float cz = __fsub_rn(__fmul_rn(e1x, e2y), __fmul_rn(e1y, e2x));
    const float len2 = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn(len2));
    const float3 ng = make_float3(__fmul_rn(cx, inv), __fmul_rn(cy, inv), __fmul_rn(cz, inv));
    is->position = make_float3(__fadd_rn(o.x, __fmul_rn(d.x, h.t)), __fadd_rn(o.y, __fmul_rn(d.y, h.t)),
                               __fadd_rn(o.z, __fmul_rn(d.z, h.t)));
    is->Ng = ng;
    is->Ns = ng;
    is->wi = make_float3(-d.x, -d.y, -d.z);
    const float dn = __fadd_rn(__fadd_rn(__fmul_rn(ng.x, d.x), __fmul_rn(ng.y, d.y)), __fmul_rn(ng.z, d.z));
    is->front = dn < 0.0f ? 1 : 0;
    is->uv = make_float2(h.u, h.v);
    is->primitive_id = (uint32_t)h.prim;
    is->primitive_material_id = tri.w;
    is->intersected = 1;
    is->epsilon = __fmul_rn(1.0e-3f, h.t);
}

// The reference's trace_ray form: fills `isect` (closest hit) or only
// isect->intersected (any hit).  Returns isect->intersected.
__device__ inline bool trace_ray(float4 o_tmin, float4 d_tmax, bool any_hit, Intersection* isect,
                                 const rb2_dev_bvh& bvh, const rb2_dev_scene& scene)
{
    rb2_hit h;
    const bool hit = trace_ray(o_tmin, d_tmax, any_hit, bvh, &h);
    if (hit && !any_hit) fill_intersection(o_tmin, d_tmax, h, scene, isect);
    isect->intersected = hit ? 1 : 0;
    return hit;
}

}  // namespace rb2
