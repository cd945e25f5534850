// Device scene, integrator scratch and the wavefront integrators (AO, path
// tracing, BDPT with a light-vertex cache).
//
// Every ray query goes through persistent_trace (rb2_traverse.cuh) with an
// integrator-specific ray source: rays are generated inside the traversal
// kernel's fetch() from path state and consumed in finish(), so secondary-ray
// buffers never round-trip through HBM.
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_internal.h"
#include "rb2_render.h"
#include "rb2_camera.cuh"
#include "rb2_film.cuh"
#include "rb2_material.cuh"
#include "rb2_shading.cuh"
#include "rb2_traverse.cuh"
#include "rb2_traverse_cw8.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

using namespace rb2;

namespace {

int cuda_fail(cudaError_t e, const char* what) { return fail(rb2::cuda_status(e), std::string(what) + ": " + cudaGetErrorString(e)); }

#define RB2_CUDA(call, what)                               \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

template <class T>
int grow(T*& p, uint64_t& cap, uint64_t n)
{
    if (n <= cap) return RB2_OK;
    rb2::dev_free(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = rb2::dev_malloc(&p, sizeof(T) * std::max<uint64_t>(n, 1));
    if (e != cudaSuccess) return fail(RB2_ENOMEM, std::string("integrator scratch: ") + cudaGetErrorString(e));
    cap = n;
    return RB2_OK;
}

}  // namespace

#include "rb2_render_internal.h"


namespace rb2dev {

using WaveCountersDev = ::WaveCounters;

// ---- AO ray source ------------------------------------------------------------------
// Slot = pixel * samples + k.  fetch() builds AO ray k of the pixel from its
// primary hit (integrators/integrator_ao.cu:51-84): origin = hit point,
// tmin = 1e-3 * t (the reference's epsilon), tmax = radius, direction
// cosine-distributed about the geometric normal facing the viewer.
struct AoSource {
    const float4* nodes;
    const float4* woop;
    const uint32_t* triidx;
    const float4* prim_rays;
    const int4* hits;
    const float4* verts;
    const uint4* tris;
    uint32_t* counts;
    unsigned long long* counter;
    uint64_t n_slots;
    uint32_t samples;
    float radius;
    uint64_t seed;
    uint32_t compat;   // RB2_COMPAT_AO_DIRECTION: the reference's direction formula

    __device__ __forceinline__ void claim(unsigned count, unsigned long long& b1, unsigned& n1, unsigned long long& b2)
    {
        b1 = atomicAdd(counter, (unsigned long long)count);
        n1 = count;
        b2 = 0;
    }

    __device__ __forceinline__ int fetch(unsigned long long slot, Lane& L) const
    {
        if (slot >= n_slots) return 0;
        const uint64_t pix = slot / samples;
        const int4 h = hits[pix];
        if (h.x < 0) return -1;
        const float t = __int_as_float(h.y);
        const float4 o4 = prim_rays[2 * pix], d4 = prim_rays[2 * pix + 1];
        const float3 pos = f3(fmaf(d4.x, t, o4.x), fmaf(d4.y, t, o4.y), fmaf(d4.z, t, o4.z));
        const uint4 tri = tris[h.x];
        const float3 v0 = xyz(verts[tri.x]), v1 = xyz(verts[tri.y]), v2 = xyz(verts[tri.z]);
        float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
        float3 dir;
        if (compat & RB2_COMPAT_AO_DIRECTION) {
            // cosine_sample_hemisphere_normal (core/montecarlo.cu:133-151) about the
            // unflipped normal; X from the cross product with the axis picked by
            // signed component comparisons.
            const float u1 = rng_u01(seed, slot, 0), u2 = rng_u01(seed, slot, 1);
            const float phi = 6.283185307179586f * u1, theta = acosf(sqrtf(1.0f - u2));
            float3 perp = f3(0.0f, 0.0f, 1.0f);
            if (ng.x < ng.y && ng.x < ng.z) perp = f3(1.0f, 0.0f, 0.0f);
            else if (ng.y < ng.x && ng.y < ng.z) perp = f3(0.0f, 1.0f, 0.0f);
            const float3 cx = cross3(ng, perp);
            const float lx2 = dot3(cx, cx);
            if (!(lx2 > 0.0f)) {  // the reference's X is NaN there: its ray never hits
                atomicAdd(&counts[pix], 1u);
                return -1;
            }
            const float3 X = mul(cx, 1.0f / sqrtf(lx2));
            const float3 Y = normalize3(cross3(ng, X));
            const float st = sinf(theta), cp = cosf(phi), sp = sinf(phi);
            dir = add(add(mul(X, cp * st), mul(Y, sp * st)), mul(ng, cp));
        } else {
            if (dot3(ng, xyz(d4)) > 0.0f) ng = mul(ng, -1.0f);
            const Frame fr = frame_from_z(ng);
            dir = to_world(fr, cosine_hemisphere(rng_u01(seed, slot, 0), rng_u01(seed, slot, 1)));
        }
        L.nodes = nodes;
        L.woop = woop;
        L.set_tag(kOcclusion, 0);
        L.ray = pix;
        setup_ray(L, make_float4(pos.x, pos.y, pos.z, 1.0e-3f * t), make_float4(dir.x, dir.y, dir.z, radius));
        return 1;
    }

    __device__ __forceinline__ void finish(const Lane& L) const
    {
        if (L.hitIndex < 0) atomicAdd(&counts[L.ray], 1u);
    }
};

// Integrator traversal: block BLOCK, register budget REGS (64: 32 warps per
// SM, 48: 40 warps), binary Compact2 or compressed 8-wide layout.
template <int BLOCK, int REGS, class Src, int LAYOUT>
__global__ void __launch_bounds__(BLOCK, (65536 / REGS) / BLOCK)
    k_persistent(Src src, uint32_t fetch_threshold, uint32_t node_threshold, unsigned int* status)
{
    if constexpr (LAYOUT == kLayoutCw8) persistent_trace_cw8<Src, true>(src, fetch_threshold, node_threshold, status);
    else persistent_trace(src, fetch_threshold, node_threshold, status);
}

__global__ void k_ao_finalize(const int4* hits, const uint32_t* counts, uint32_t npix, uint32_t samples, float* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x)
        out[i] = hits[i].x >= 0 ? (float)counts[i] / (float)samples : 0.0f;
}

// ---- path tracing -----------------------------------------------------------------
// Random dimensions per (sample key, vertex b): camera jitter uses dims 0-1,
// vertex b uses 8 dims from 2 + 8b.
enum : uint32_t { kDimLight = 0, kDimLightU = 1, kDimLightV = 2, kDimBsdfU = 3, kDimBsdfV = 4, kDimRR = 5,
                  kDimBsdfC = 6 };
__device__ __forceinline__ uint32_t vdim(uint32_t b, uint32_t d) { return 2u + 8u * b + d; }

struct SceneView {
    const float4* verts;
    const uint4* tris;
    const float4* albedo;
    const float4* emission;
    const uint32_t* lights;
    uint32_t n_lights;
    const MaterialDev* mats;   // null: every material is one Lambertian layer (albedo)
};

// Queue-driven ray source: the i-th entry of `queue` names a path whose ray
// is in `rays`; `n` (device) is the queue length written by the previous
// kernel, so no host round trip is needed between stages.
struct QueueSource {
    const float4* nodes;
    const float4* woop;
    const uint32_t* triidx;
    const uint32_t* queue;
    const uint32_t* n;
    const float4* rays;
    unsigned long long* head;
    uint32_t mode;
    // closest hit: store the hit record; occlusion: add the pending contribution
    // to L when unoccluded, or (L == nullptr) clear `contrib` when occluded
    int4* hits;
    float4* L;
    float4* contrib;

    __device__ __forceinline__ void claim(unsigned count, unsigned long long& b1, unsigned& n1, unsigned long long& b2)
    {
        b1 = atomicAdd(head, (unsigned long long)count);
        n1 = count;
        b2 = 0;
    }

    __device__ __forceinline__ int fetch(unsigned long long slot, Lane& L_) const
    {
        if (slot >= (unsigned long long)__ldg(n)) return 0;
        const uint32_t path = __ldg(queue + slot);
        L_.nodes = nodes;
        L_.woop = woop;
        L_.set_tag(mode, 0);
        L_.ray = path;
        setup_ray(L_, rays[2 * (size_t)path], rays[2 * (size_t)path + 1]);
        return 1;
    }

    __device__ __forceinline__ void finish(const Lane& L_) const
    {
        if (mode == kClosest) {
            hits[L_.ray] = hit_record(L_, triidx);
        } else if (L == nullptr) {
            if (L_.hitIndex >= 0) contrib[L_.ray] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else if (L_.hitIndex < 0) {
            const float4 c = contrib[L_.ray];
            float4 a = L[L_.ray];
            L[L_.ray] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w);
        }
    }
};

// Warp-aggregated append: returns this lane's slot (valid only when pred).
__device__ __forceinline__ uint32_t warp_append(uint32_t* count, bool pred)
{
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, pred);
    if (!m) return 0;
    const int leader = __ffs(m) - 1;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(act, base, leader);
    return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

__global__ void k_pt_camera(CamArgs cam, uint64_t seed, uint32_t npix, uint32_t paths, uint32_t sample0,
                            float4* rays, float4* T, float4* L, uint32_t* q0, WaveCountersDev* wc,
                            float2* xy_out = nullptr)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wc->n_ext[0] = paths;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
        const uint32_t pix = p % npix;
        const uint64_t key = (uint64_t)(sample0 + p / npix) * npix + pix;
        const float jx = rng_u01(seed, key, 0), jy = rng_u01(seed, key, 1);
        float4 o, d;
        const float sx = (float)(pix % cam.width) + jx, sy = (float)(pix / cam.width) + jy;
        camera_ray(cam.r2c, cam.c2w, sx, sy, o, d);
        if (xy_out) xy_out[p] = make_float2(sx, sy);
        rays[2 * (size_t)p] = o;
        rays[2 * (size_t)p + 1] = d;
        if (T) T[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);  // null: no path state (ray casting)
        if (L) L[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        q0[p] = p;
    }
}

__global__ void k_pt_bounce_reset(WaveCountersDev* wc, uint32_t next)
{
    wc->n_ext[next] = 0;
    wc->n_shadow = 0;
    wc->n_conn = 0;
    wc->head_ext = 0;
    wc->head_shadow = 0;
    wc->head_conn = 0;
}

__device__ __forceinline__ float tri_area(float3 v0, float3 v1, float3 v2)
{
    return 0.5f * sqrtf(dot3(cross3(sub(v1, v0), sub(v2, v0)), cross3(sub(v1, v0), sub(v2, v0))));
}

// Shade every path of the current queue at vertex b (integrator_path.cu:84-254):
// emission (MIS-weighted after the first vertex), next-event estimation with
// a shadow ray, BSDF sampling of the continuation, Russian roulette.
// Path vertex on a layered material (core/material.cu, core/reflection.cu):
// next-event estimation with material_f / material_pdf (skipped for purely
// specular materials), then material_sample_f for the continuation.  T.w
// carries the sampled pdf for the emission MIS weight, -1 after a specular
// bounce (full weight, as integrator_path.cu:94 counts emission after one).
// Russian roulette of a camera path after the BSDF sample at vertex b: from
// b = rr_start with division by q, or (RB2_COMPAT_RR_DIVISOR) from
// b = rr_start + 1 with division by 1 - q (integrator_path.cu:232-244).
__device__ __forceinline__ bool roulette(float4& Tp, uint32_t b, uint32_t rr_start, float rr_prob, uint32_t compat,
                                         float u)
{
    const bool ref = (compat & RB2_COMPAT_RR_DIVISOR) != 0;
    if (ref ? b <= rr_start : b < rr_start) return true;
    const float q = fminf(rr_prob, luminance(xyz(Tp)));
    if (!(u < q)) return false;
    const float inv = ref ? 1.0f / (1.0f - q) : 1.0f / q;
    Tp.x *= inv; Tp.y *= inv; Tp.z *= inv;
    return true;
}

__device__ __forceinline__ void shade_layered(const SceneView& sc, const MaterialDev& m, uint64_t seed, uint64_t key,
                                              uint32_t b, uint32_t max_depth, uint32_t rr_start, float rr_prob,
                                              uint32_t compat, float inv_nl, float3 pos, float eps, float3 ng,
                                              float3 wo, float4& Tp, bool& shadow, float4& so, float4& sd,
                                              float4& scv, bool& cont, float4& new_o, float4& new_d)
{
    const Frame fr = frame_from_z(ng);
    const float3 wo_l = to_local(fr, wo);
    const uint32_t bn = (compat & RB2_COMPAT_NEE_RESEED) ? 0u : b;  // NEE draws of this vertex
    if (sc.n_lights && (m.flags & kMatHasNonDelta)) {
        uint32_t j = (uint32_t)(rng_u01(seed, key, vdim(bn, kDimLight)) * (float)sc.n_lights);
        j = min(j, sc.n_lights - 1);
        const uint4 lt = sc.tris[sc.lights[j]];
        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
        const float3 lp = sample_triangle(l0, l1, l2, rng_u01(seed, key, vdim(bn, kDimLightU)),
                                          rng_u01(seed, key, vdim(bn, kDimLightV)));
        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
        const float3 dv = sub(lp, pos);
        const float dist2 = dot3(dv, dv);
        const float dist = sqrtf(dist2);
        const float3 wi = mul(dv, 1.0f / dist);
        const float cos_l = -dot3(ln, wi);
        if (cos_l > 0.0f && dist > 0.0f) {
            const float3 wi_l = to_local(fr, wi);
            const float3 f = material_f(m, ng, wo, wi, wo_l, wi_l);
            if (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f) {
                const float4 Le = sc.emission[lt.w];
                const float pdf_l = inv_nl * dist2 / (tri_area(l0, l1, l2) * cos_l);
                const float pdf_b = material_pdf(m, wo_l, wi_l);
                const float w = (b == max_depth) ? 1.0f : pdf_l / (pdf_l + pdf_b);
                const float k = fabsf(dot3(wi, ng)) * w / pdf_l;
                scv = make_float4(Tp.x * f.x * Le.x * k, Tp.y * f.y * Le.y * k, Tp.z * f.z * Le.z * k, 0.0f);
                so = make_float4(pos.x, pos.y, pos.z, eps);
                sd = make_float4(wi.x, wi.y, wi.z, dist * (1.0f - 1.0e-3f));
                shadow = scv.x > 0.0f || scv.y > 0.0f || scv.z > 0.0f;
            }
        }
    }
    if (b >= max_depth) return;
    float3 wi;
    float pdf;
    bool spec;
    const float3 f = material_sample(m, fr, ng, wo, rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                     rng_u01(seed, key, vdim(b, kDimBsdfV)), rng_u01(seed, key, vdim(b, kDimBsdfC)), wi,
                                     pdf, spec);
    if (!(pdf > 0.0f) || !(f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) return;
    const float k = fabsf(dot3(wi, ng)) / pdf;
    Tp.x *= f.x * k; Tp.y *= f.y * k; Tp.z *= f.z * k;
    Tp.w = spec ? -1.0f : pdf;
    cont = isfinite(Tp.x) && isfinite(Tp.y) && isfinite(Tp.z) && (Tp.x > 0.0f || Tp.y > 0.0f || Tp.z > 0.0f);
    if (cont) cont = roulette(Tp, b, rr_start, rr_prob, compat, rng_u01(seed, key, vdim(b, kDimRR)));
    if (cont) {
        new_o = make_float4(pos.x, pos.y, pos.z, eps);
        new_d = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
    }
}

__global__ void k_pt_shade(SceneView sc, uint64_t seed, uint32_t npix, uint32_t sample0, uint32_t b, uint32_t max_depth,
                           uint32_t rr_start, float rr_prob, uint32_t compat, const uint32_t* q_in, uint32_t* q_out,
                           float4* rays,
                           const int4* hits, float4* T, float4* L, float4* srays, float4* sc_out, uint32_t* qs,
                           WaveCountersDev* wc, uint32_t cur)
{
    const uint32_t n = wc->n_ext[cur];
    const uint32_t next = cur ^ 1u;
    const float inv_nl = sc.n_lights ? 1.0f / (float)sc.n_lights : 0.0f;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool cont = false, shadow = false;
        uint32_t path = 0;
        float4 new_o, new_d, so, sd, scv;
        if (i < n) {
            path = q_in[i];
            const int4 h = hits[path];
            if (h.x >= 0) {
                const uint32_t pix = path % npix;
                const uint64_t key = (uint64_t)(sample0 + path / npix) * npix + pix;
                const float4 o4 = rays[2 * (size_t)path], d4 = rays[2 * (size_t)path + 1];
                const float t = __int_as_float(h.y);
                const float3 d = xyz(d4);
                const float3 pos = f3(fmaf(d.x, t, o4.x), fmaf(d.y, t, o4.y), fmaf(d.z, t, o4.z));
                const float eps = 1.0e-3f * t;
                const uint4 tri = sc.tris[h.x];
                const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
                const float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
                const float3 wo = mul(d, -1.0f);
                float4 Tp = T[path];
                const float4 E = sc.emission[tri.w];
                if (E.x > 0.0f || E.y > 0.0f || E.z > 0.0f) {
                    // DiffuseAreaLight::L (core/lights.cu:70-78): one-sided emitter.
                    const float cosl = dot3(ng, wo);
                    if (cosl > 0.0f) {
                        float4 Lp = L[path];  // read only where a path gains emission
                        float w = 1.0f;
                        if (b > 0 && Tp.w > 0.0f) {  // T.w < 0: the last bounce was specular
                            const float pdf_l = inv_nl * t * t / (tri_area(v0, v1, v2) * cosl);
                            w = Tp.w / (Tp.w + pdf_l);
                        }
                        Lp.x += Tp.x * E.x * w; Lp.y += Tp.y * E.y * w; Lp.z += Tp.z * E.z * w;
                        L[path] = Lp;
                    }
                    // Emitters end the path (integrator_path.cu:94-107).
                } else if (sc.mats != nullptr && !(sc.mats[tri.w].flags & kMatPlainLambertian)) {
                    shade_layered(sc, sc.mats[tri.w], seed, key, b, max_depth, rr_start, rr_prob, compat, inv_nl, pos,
                                  eps, ng, wo, Tp, shadow, so, sd, scv, cont, new_o, new_d);
                    if (cont) T[path] = Tp;
                } else {
                    const float3 nrm = dot3(ng, wo) < 0.0f ? mul(ng, -1.0f) : ng;
                    const float4 A = sc.albedo[tri.w];
                    // Next-event estimation to one uniformly chosen emissive triangle.
                    if (sc.n_lights) {
                        const uint32_t bn = (compat & RB2_COMPAT_NEE_RESEED) ? 0u : b;
                        uint32_t j = (uint32_t)(rng_u01(seed, key, vdim(bn, kDimLight)) * (float)sc.n_lights);
                        j = min(j, sc.n_lights - 1);
                        const uint4 lt = sc.tris[sc.lights[j]];
                        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
                        const float3 lp = sample_triangle(l0, l1, l2, rng_u01(seed, key, vdim(bn, kDimLightU)),
                                                          rng_u01(seed, key, vdim(bn, kDimLightV)));
                        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
                        const float3 dv = sub(lp, pos);
                        const float dist2 = dot3(dv, dv);
                        const float dist = sqrtf(dist2);
                        const float3 wi = mul(dv, 1.0f / dist);
                        const float cos_l = -dot3(ln, wi);
                        const float cos_s = dot3(nrm, wi);
                        const float4 Le = sc.emission[lt.w];
                        if (cos_l > 0.0f && cos_s > 0.0f && dist > 0.0f) {
                            const float pdf_l = inv_nl * dist2 / (tri_area(l0, l1, l2) * cos_l);
                            const float pdf_b = cos_s * kInvPi;
                            const float w = (b == max_depth) ? 1.0f : pdf_l / (pdf_l + pdf_b);
                            const float k = cos_s * w / pdf_l * kInvPi;
                            scv = make_float4(Tp.x * A.x * Le.x * k, Tp.y * A.y * Le.y * k, Tp.z * A.z * Le.z * k, 0.0f);
                            // VisibilityTesterElement::set_segment (core/util.h:186-195).
                            so = make_float4(pos.x, pos.y, pos.z, eps);
                            sd = make_float4(wi.x, wi.y, wi.z, dist * (1.0f - 1.0e-3f));
                            shadow = scv.x > 0.0f || scv.y > 0.0f || scv.z > 0.0f;
                        }
                    }
                    if (b < max_depth) {
                        // Lambertian sample (core/reflection.cu:42-69): f cos / pdf = albedo.
                        const float3 loc = cosine_hemisphere(rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                                             rng_u01(seed, key, vdim(b, kDimBsdfV)));
                        const float pdf = loc.z * kInvPi;
                        if (pdf > 0.0f) {
                            const float3 wi = normalize3(to_world(frame_from_z(nrm), loc));
                            Tp.x *= A.x; Tp.y *= A.y; Tp.z *= A.z; Tp.w = pdf;
                            cont = Tp.x > 0.0f || Tp.y > 0.0f || Tp.z > 0.0f;
                            // Unbiased Russian roulette unless RB2_COMPAT_RR_DIVISOR asks for
                            // the reference's division by 1 - q (integrator_path.cu:232-244).
                            if (cont) cont = roulette(Tp, b, rr_start, rr_prob, compat, rng_u01(seed, key, vdim(b, kDimRR)));
                            if (cont) {
                                T[path] = Tp;
                                new_o = make_float4(pos.x, pos.y, pos.z, eps);
                                new_d = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    }
                }
            }
        }
        const uint32_t so_slot = warp_append(&wc->n_shadow, shadow);
        if (shadow) {
            srays[2 * (size_t)path] = so;
            srays[2 * (size_t)path + 1] = sd;
            sc_out[path] = scv;
            qs[so_slot] = path;
        }
        const uint32_t ext_slot = warp_append(&wc->n_ext[next], cont);
        if (cont) {
            rays[2 * (size_t)path] = new_o;
            rays[2 * (size_t)path + 1] = new_d;
            q_out[ext_slot] = path;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&wc->stats[b == 0 ? 0 : 1], (unsigned long long)n);
    }
}

__global__ void k_pt_stats_shadow(WaveCountersDev* wc)
{
    wc->stats[2] += wc->n_shadow;
}

__global__ void k_pt_accumulate(const float4* L, uint32_t npix, uint32_t per_pixel, float4* accum)
{
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        float4 a = accum[pix];
        for (uint32_t j = 0; j < per_pixel; j++) {
            const float4 l = L[(size_t)j * npix + pix];
            a.x += l.x; a.y += l.y; a.z += l.z;
        }
        accum[pix] = a;
    }
}

// ---- Ray casting (integrators/integrator_raycast.cu:27-113) ---------------------------
// The reference's palette for primitive ids (its entries, in its order; the
// names in its comments do not all match the values).
__constant__ float4 kRayCastPalette[15] = {
    {1.0f, 0.0f, 0.0f, 0.0f},   {0.0f, 1.0f, 0.0f, 0.0f},  {0.0f, 0.0f, 1.0f, 0.0f}, {0.0f, 1.0f, 1.0f, 0.0f},
    {1.0f, 0.0f, 1.0f, 0.0f},   {1.0f, 1.0f, 0.0f, 0.0f},  {0.1f, 0.1f, 0.1f, 0.0f}, {0.5f, 0.5f, 0.5f, 0.0f},
    {1.0f, 1.0f, 1.0f, 0.0f},   {0.0f, 0.25f, 0.5f, 0.0f}, {1.0f, 0.5f, 0.0f, 0.0f}, {0.5f, 0.25f, 0.0f, 0.0f},
    {0.2f, 0.9f, 1.0f, 0.0f},   {0.7f, 0.3f, 0.1f, 0.0f},  {0.34f, 0.89f, 0.45f, 0.0f}};

// The colour of one camera sample from its closest hit (kernel_ray_cast_update):
// mode is an RB2_RAYCAST_SHADE_* value; misses stay black in every mode.
__device__ __forceinline__ float3 rc_colour(const SceneView& sc, int h, uint32_t mode)
{
    float3 c = f3(0.0f, 0.0f, 0.0f);
    if (h < 0) return c;
    if (mode == RB2_RAYCAST_SHADE_PRIMITIVE_ID) {
        c = xyz(kRayCastPalette[(uint32_t)h % 15u]);
    } else if (mode == RB2_RAYCAST_SHADE_MATERIAL_ID) {
        // First layer's colour; an emitter shows its emission.
        const uint32_t m = sc.tris[h].w;
        const float4 E = sc.emission[m];
        if (E.x > 0.0f || E.y > 0.0f || E.z > 0.0f) {
            c = xyz(E);
        } else if (sc.mats && !(sc.mats[m].flags & kMatPlainLambertian)) {
            const LayerDev& l = sc.mats[m].layer[0];
            if (layer_kind(l) != kOrenNayar) c = xyz(l.q0);
        } else {
            c = xyz(sc.albedo[m]);
        }
    } else if (mode == RB2_RAYCAST_SHADE_NORMALS) {
        const uint4 tri = sc.tris[h];
        const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
        c = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
    } else if (mode == RB2_RAYCAST_SHADE_UNIFORM) {
        c = f3(1.0f, 1.0f, 1.0f);
    }
    return c;
}

// Per-sample colours into L (the film gather reads them with the sample positions).
__global__ void k_rc_shade(SceneView sc, uint32_t paths, uint32_t mode, const int4* hits, float4* L,
                           WaveCountersDev* wc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wc->stats[0] += paths;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
        const float3 c = rc_colour(sc, hits[p].x, mode);
        L[p] = make_float4(c.x, c.y, c.z, 0.0f);
    }
}

// Unfiltered: shade a pixel's samples of the wave in sample order and add them
// to its accumulator (the sums k_rc_shade + k_pt_accumulate form, without the
// per-sample colour buffer).
__global__ void k_rc_shade_accumulate(SceneView sc, uint32_t npix, uint32_t per_pixel, uint32_t mode,
                                      const int4* hits, float4* accum, WaveCountersDev* wc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wc->stats[0] += (unsigned long long)npix * per_pixel;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        float4 a = accum[pix];
        for (uint32_t j = 0; j < per_pixel; j++) {
            const float3 c = rc_colour(sc, hits[(size_t)j * npix + pix].x, mode);
            a.x += c.x; a.y += c.y; a.z += c.z;
        }
        accum[pix] = a;
    }
}

// ---- BDPT with a light-vertex cache -----------------------------------------------
constexpr uint32_t kMaxConnections = 8;
constexpr uint64_t kLightSalt = 0xA24BAED4963EE407ull;
constexpr float kLightRayTmin = 1.0e-4f;

// ---- Strategy counting with specular vertices.  A path of k segments
// x_1..x_k (x_k on a light) can be sampled by strategy s = 0 (the camera
// subpath hits the light) and, for each edge (x_j, x_j+1), j = 1..k-1, by the
// connection across it, which is possible only when neither endpoint scatters
// specularly on this path (f at a connection vertex is the non-specular part).
// Every possible strategy is weighted 1 / n_valid, n_valid = 1 + (edges whose
// endpoints both scatter non-specularly), which is k when no vertex is
// specular.  A subpath carries the count of valid edges so far and whether its
// last vertex scattered non-specularly, packed in one word.
__device__ __forceinline__ uint32_t bd_state(uint32_t nonspec_prev, uint32_t edges) { return nonspec_prev | (edges << 1); }
__device__ __forceinline__ uint32_t bd_edges(uint32_t st) { return st >> 1; }
__device__ __forceinline__ uint32_t bd_nonspec(uint32_t st) { return st & 1u; }
// After a vertex that scattered (non-)specularly.
__device__ __forceinline__ uint32_t bd_advance(uint32_t st, bool nonspec)
{
    return bd_state(nonspec ? 1u : 0u, bd_edges(st) + (bd_nonspec(st) && nonspec ? 1u : 0u));
}

// Light subpath start (integrators/integrator_bdpt_lvc_sk.cu:61-83): uniform
// emissive triangle, uniform point, cosine-distributed direction about its
// normal (one-sided emitter).  Throughput Le cos / (pdf_A pdf_w) = Le NL A pi.
__global__ void k_bd_light_init(SceneView sc, uint64_t seed, uint64_t key0, uint32_t n_paths, float4* lray,
                                float4* lbeta, uint32_t* lq0, WaveCountersDev* wc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wc->n_ext[0] = sc.n_lights ? n_paths : 0u;
    if (!sc.n_lights) return;
    const uint64_t ls = seed ^ kLightSalt;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_paths; p += gridDim.x * blockDim.x) {
        const uint64_t key = key0 + p;
        uint32_t j = min((uint32_t)(rng_u01(ls, key, 0) * (float)sc.n_lights), sc.n_lights - 1);
        const uint4 lt = sc.tris[sc.lights[j]];
        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
        const float3 y0 = sample_triangle(l0, l1, l2, rng_u01(ls, key, 1), rng_u01(ls, key, 2));
        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
        const float3 dir = normalize3(to_world(frame_from_z(ln), cosine_hemisphere(rng_u01(ls, key, 3), rng_u01(ls, key, 4))));
        const float4 Le = sc.emission[lt.w];
        const float k = (float)sc.n_lights * tri_area(l0, l1, l2) * 3.14159265358979f;
        // w: strategy bookkeeping (non-specular previous vertex, valid edges so far);
        // the light point itself is non-specular.
        lbeta[p] = make_float4(Le.x * k, Le.y * k, Le.z * k, __uint_as_float(bd_state(1u, 0u)));
        lray[2 * (size_t)p] = make_float4(y0.x, y0.y, y0.z, kLightRayTmin);
        lray[2 * (size_t)p + 1] = make_float4(dir.x, dir.y, dir.z, 3.402823466e+38f);
        lq0[p] = p;
    }
}

// Layered material of a surface, or null for a single Lambertian layer (the
// albedo fast path).
__device__ __forceinline__ const MaterialDev* layered_material(const SceneView& sc, uint32_t mat)
{
    return (sc.mats && !(sc.mats[mat].flags & kMatPlainLambertian)) ? &sc.mats[mat] : nullptr;
}

// Light vertex d (1-based surface vertex): store it in the sparse cache slot
// (path, d) and continue the subpath by BSDF sampling with Russian roulette on
// the per-bounce factor (integrator_bdpt_lvc_sk.cu:93-166).  On a layered
// material the continuation samples material_sample_f and the factor is
// f |cos| / pdf (f the adjoint); s_wi (null when every material is one
// Lambertian layer) keeps the direction toward the previous vertex for the
// connection's f.
__global__ void k_bd_light_shade(SceneView sc, uint64_t seed, uint64_t key0, uint32_t d, uint32_t Dl, uint32_t rr_start,
                                 float rr_prob, const uint32_t* q_in, uint32_t* q_out, float4* lray, const int4* lhit,
                                 float4* lbeta, float4* s_pos, float4* s_nrm, float4* s_beta, float4* s_wi,
                                 uint8_t* s_valid, WaveCountersDev* wc, uint32_t cur)
{
    const uint32_t n = wc->n_ext[cur];
    const uint64_t ls = seed ^ kLightSalt;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool cont = false;
        uint32_t path = 0;
        float4 no, nd;
        if (i < n) {
            path = q_in[i];
            const int4 h = lhit[path];
            if (h.x >= 0) {
                const float4 o4 = lray[2 * (size_t)path], d4 = lray[2 * (size_t)path + 1];
                const float t = __int_as_float(h.y);
                const float3 dd = xyz(d4);
                const float3 pos = f3(fmaf(dd.x, t, o4.x), fmaf(dd.y, t, o4.y), fmaf(dd.z, t, o4.z));
                const uint4 tri = sc.tris[h.x];
                const float4 E = sc.emission[tri.w];
                if (!(E.x > 0.0f || E.y > 0.0f || E.z > 0.0f)) {
                    const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
                    const float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
                    const float3 wo = mul(dd, -1.0f);
                    const float3 nrm = dot3(ng, wo) < 0.0f ? mul(ng, -1.0f) : ng;
                    float4 beta = lbeta[path];
                    const uint32_t st = __float_as_uint(beta.w);
                    const size_t slot = (size_t)path * Dl + (d - 1);
                    const MaterialDev* lm = layered_material(sc, tri.w);
                    // A vertex whose material is purely specular cannot be connected to:
                    // it is not cached.  The cached w is the light side's valid-edge count
                    // with this vertex as a (non-specular) connection endpoint.
                    if (!lm || (lm->flags & kMatHasNonDelta)) {
                        s_pos[slot] = make_float4(pos.x, pos.y, pos.z, (float)(d + 1));
                        s_nrm[slot] = make_float4(nrm.x, nrm.y, nrm.z, __uint_as_float(tri.w));
                        s_beta[slot] = make_float4(beta.x, beta.y, beta.z, (float)(bd_edges(st) + bd_nonspec(st)));
                        s_valid[slot] = 1;
                        if (s_wi) s_wi[slot] = make_float4(wo.x, wo.y, wo.z, dot3(ng, nrm) < 0.0f ? -1.0f : 1.0f);
                    }
                    if (d < Dl && lm) {
                        const uint64_t key = key0 + path;
                        float3 wi;
                        float pdf, eta_io;
                        bool spec;
                        const Frame frl = frame_from_z(ng);
                        float3 f = material_sample(*lm, frl, ng, wo, rng_u01(ls, key, 8 + 8 * d),
                                                   rng_u01(ls, key, 9 + 8 * d), rng_u01(ls, key, 11 + 8 * d), wi, pdf, spec,
                                                   &eta_io);
                        if (pdf > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) {
                            if (!spec) {
                                // Light flows from wo toward wi: the adjoint f(wi -> wo), since the
                                // Blinn shadowing term is not symmetric in its two directions.
                                f = material_f(*lm, ng, wi, wo, to_local(frl, wi), to_local(frl, wo));
                            } else if (eta_io != 1.0f) {
                                // Adjoint of the glass transmission: the camera-side factor
                                // carries (eta of wi / eta of wo)^2, and the refraction maps
                                // solid angle by (eta_o / eta_i)^2 cos_o / cos_i, so the factor
                                // seen from the light is the sampled one times eta_io^6.
                                const float e2 = eta_io * eta_io, e6 = e2 * e2 * e2;
                                f = f3(f.x * e6, f.y * e6, f.z * e6);
                            }
                            const float k = fabsf(dot3(wi, ng)) / pdf;
                            const float3 fac = f3(f.x * k, f.y * k, f.z * k);
                            float q = fminf(1.0f, luminance(fac));
                            if (d < rr_start) q = 1.0f;
                            else q = fminf(q, rr_prob);
                            cont = q > 0.0f && isfinite(fac.x) && isfinite(fac.y) && isfinite(fac.z) &&
                                   rng_u01(ls, key, 10 + 8 * d) < q;
                            if (cont) {
                                beta.x *= fac.x / q; beta.y *= fac.y / q; beta.z *= fac.z / q;
                                beta.w = __uint_as_float(bd_advance(st, !spec));
                                lbeta[path] = beta;
                                no = make_float4(pos.x, pos.y, pos.z, 1.0e-3f * t);
                                nd = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    } else if (d < Dl) {
                        const uint64_t key = key0 + path;
                        const float4 A = sc.albedo[tri.w];
                        const float3 loc = cosine_hemisphere(rng_u01(ls, key, 8 + 8 * d), rng_u01(ls, key, 9 + 8 * d));
                        if (loc.z > 0.0f) {
                            const float3 wi = normalize3(to_world(frame_from_z(nrm), loc));
                            float q = fminf(1.0f, luminance(xyz(A)));
                            if (d < rr_start) q = 1.0f;
                            else q = fminf(q, rr_prob);
                            cont = q > 0.0f && rng_u01(ls, key, 10 + 8 * d) < q;
                            if (cont) {
                                beta.x *= A.x / q; beta.y *= A.y / q; beta.z *= A.z / q;
                                beta.w = __uint_as_float(bd_advance(st, true));
                                lbeta[path] = beta;
                                no = make_float4(pos.x, pos.y, pos.z, 1.0e-3f * t);
                                nd = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    }
                }
            }
        }
        const uint32_t slot_out = warp_append(&wc->n_ext[cur ^ 1u], cont);
        if (cont) {
            lray[2 * (size_t)path] = no;
            lray[2 * (size_t)path + 1] = nd;
            q_out[slot_out] = path;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&wc->stats[4], (unsigned long long)n);
}

// Deterministic cache compaction: chunks of kScanChunk sparse slots.
constexpr uint32_t kScanChunk = 2048;
constexpr uint32_t kScanThreads = 256;

__global__ void k_lvc_count(const uint8_t* valid, uint64_t n_slots, uint32_t* block_sums)
{
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < kScanChunk; k += kScanThreads) {
        const uint64_t i = base + k;
        if (i < n_slots) c += valid[i];
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t w = 0; w < kScanThreads / 32; w++) t += s_warp[w];
        block_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the per-chunk counts in one block; total -> lvc_count.
__global__ void k_lvc_scan_top(uint32_t* block_sums, uint32_t n_blocks, WaveCountersDev* wc)
{
    __shared__ uint32_t s[1024];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n_blocks; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n_blocks ? block_sums[i] : 0u;
        s[threadIdx.x] = v;
        __syncthreads();
        for (uint32_t off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
            const uint32_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
            __syncthreads();
            s[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < n_blocks) block_sums[i] = carry + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        wc->lvc_count = carry;
        wc->stats[5] += carry;
    }
}

// Dense list of the valid slots, in slot order: a chunk is read in rounds of
// kScanThreads consecutive slots (coalesced flags, coalesced index writes); a
// round's valid slots go after the chunk's offset and the earlier rounds'.
// Connections read the sparse cache through this list, so no vertex data is
// copied.
__global__ void k_lvc_scatter(const uint8_t* valid, uint64_t n_slots, const uint32_t* block_offsets, uint32_t* slot_of)
{
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t run = block_offsets[blockIdx.x];
    for (uint32_t r = 0; r < kScanChunk / kScanThreads; r++) {
        const uint64_t i = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)r * kScanThreads + threadIdx.x;
        const bool v = i < n_slots && valid[i] != 0;
        const unsigned m = __ballot_sync(kFull, v);
        if (lane == 0) s_warp[warp] = (uint32_t)__popc(m);
        __syncthreads();
        uint32_t off = run, tot = 0;
        for (uint32_t w = 0; w < kScanThreads / 32; w++) {
            if (w < warp) off += s_warp[w];
            tot += s_warp[w];
        }
        if (v) slot_of[off + (uint32_t)__popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
        run += tot;
        __syncthreads();  // s_warp is rewritten by the next round
    }
}

// Dense-cache offset of each iteration of a wave: the valid slots before slot
// i x per_iter (i = 0..w), the scan's offset of the boundary's chunk plus a
// count inside that chunk.  One block per boundary; a boundary at or past the
// end gets the total.
__global__ void k_lvc_wave_offsets(const uint8_t* valid, uint64_t n_slots, const uint32_t* block_offsets,
                                   uint64_t per_iter, const WaveCountersDev* wc, uint32_t* lvc_off)
{
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const uint64_t b = (uint64_t)blockIdx.x * per_iter;
    if (b >= n_slots) {  // uniform over the block
        if (threadIdx.x == 0) lvc_off[blockIdx.x] = wc->lvc_count;
        return;
    }
    const uint64_t chunk = b / kScanChunk;
    uint32_t c = 0;
    for (uint64_t k = chunk * kScanChunk + threadIdx.x; k < b; k += kScanThreads) c += valid[k];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (uint32_t w = 0; w < kScanThreads / 32; w++) tot += s_warp[w];
        lvc_off[blockIdx.x] = block_offsets[chunk] + tot;
    }
}

// Camera vertex i (1-based): emission (s = 0), next-event estimation (s = 1),
// connections to cached light vertices (s >= 2), continuation.  Every
// strategy of a path is weighted 1/n_valid (the strategy counting above).  A
// layered vertex at either end of a connection takes f from material_f in the frame of
// its geometric normal (the path tracer's convention) and continues by
// material_sample_f; single-Lambertian vertices keep the albedo fast path.
__global__ void k_bd_cam_shade(SceneView sc, uint64_t seed, uint32_t npix, uint32_t it0, uint32_t i, uint32_t Kmax,
                               uint32_t C, uint32_t rr_start, float rr_prob, float n_light_paths, const uint32_t* q_in,
                               uint32_t* q_out, float4* rays, const int4* hits, float4* T, float4* L, float4* srays,
                               float4* sc_out, uint32_t* qs, float4* cray, float4* cc, uint32_t* cq,
                               const float4* lvc_pos, const float4* lvc_nrm, const float4* lvc_beta,
                               const float4* lvc_wi, const uint32_t* lvc_slot, const uint32_t* lvc_off,
                               WaveCountersDev* wc, uint32_t cur)
{
    const uint32_t n = wc->n_ext[cur];
    const float inv_nl = sc.n_lights ? 1.0f / (float)sc.n_lights : 0.0f;
    const uint32_t b = i - 1;  // random-dimension block of this vertex
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t qi = base + threadIdx.x;
        bool cont = false, shadow = false;
        bool conn[kMaxConnections];
        float4 cro[kMaxConnections], crd[kMaxConnections];
        for (uint32_t c = 0; c < kMaxConnections; c++) conn[c] = false;
        uint32_t path = 0;
        float4 new_o, new_d, so, sd, scv;
        if (qi < n) {
            path = q_in[qi];
            for (uint32_t c = 0; c < C; c++) cc[(size_t)path * C + c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const int4 h = hits[path];
            if (h.x >= 0) {
                // Path p of the wave is pixel p % npix of iteration it0 + p / npix, whose
                // cached light vertices are the dense range [lvc_off[li], lvc_off[li + 1]).
                const uint64_t key = (uint64_t)it0 * npix + path;
                const uint32_t li = path / npix;
                const uint32_t vbase = lvc_off[li], M = lvc_off[li + 1] - vbase;
                const float4 o4 = rays[2 * (size_t)path], d4 = rays[2 * (size_t)path + 1];
                const float t = __int_as_float(h.y);
                const float3 d = xyz(d4);
                const float3 pos = f3(fmaf(d.x, t, o4.x), fmaf(d.y, t, o4.y), fmaf(d.z, t, o4.z));
                const float eps = 1.0e-3f * t;
                const uint4 tri = sc.tris[h.x];
                const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
                const float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
                const float3 wo = mul(d, -1.0f);
                float4 Tp = T[path];
                // Valid-edge count of the camera subpath before this vertex, plus the
                // edge to it when the previous vertex scattered non-specularly (the
                // camera itself counts as specular: T.w starts at 0).
                const uint32_t cst = __float_as_uint(Tp.w);
                const uint32_t cbase = bd_edges(cst) + bd_nonspec(cst);
                const float4 E = sc.emission[tri.w];
                if (E.x > 0.0f || E.y > 0.0f || E.z > 0.0f) {
                    if (dot3(ng, wo) > 0.0f) {  // s = 0, k = i
                        float4 Lp = L[path];
                        const float w = 1.0f / (float)(1u + cbase);  // s = 0
                        Lp.x += Tp.x * E.x * w; Lp.y += Tp.y * E.y * w; Lp.z += Tp.z * E.z * w;
                        L[path] = Lp;
                    }
                } else {
                    const float3 nrm = dot3(ng, wo) < 0.0f ? mul(ng, -1.0f) : ng;
                    const float4 A = sc.albedo[tri.w];
                    const MaterialDev* mc = layered_material(sc, tri.w);
                    const Frame frc = frame_from_z(ng);
                    const float3 wo_l = to_local(frc, wo);
                    if (sc.n_lights && i + 1 <= Kmax) {  // s = 1, k = i + 1
                        uint32_t j = min((uint32_t)(rng_u01(seed, key, vdim(b, kDimLight)) * (float)sc.n_lights),
                                         sc.n_lights - 1);
                        const uint4 lt = sc.tris[sc.lights[j]];
                        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
                        const float3 lp = sample_triangle(l0, l1, l2, rng_u01(seed, key, vdim(b, kDimLightU)),
                                                          rng_u01(seed, key, vdim(b, kDimLightV)));
                        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
                        const float3 dv = sub(lp, pos);
                        const float dist2 = dot3(dv, dv), dist = sqrtf(dist2);
                        const float3 wi = mul(dv, 1.0f / dist);
                        const float cos_l = -dot3(ln, wi), cos_s = dot3(nrm, wi);
                        const float4 Le = sc.emission[lt.w];
                        if (mc && cos_l > 0.0f && dist > 0.0f) {
                            const float3 f = material_f(*mc, ng, wo, wi, wo_l, to_local(frc, wi));
                            const float pdf_l = inv_nl * dist2 / (tri_area(l0, l1, l2) * cos_l);
                            const float k = fabsf(cos_s) / (pdf_l * (float)(2u + cbase));
                            scv = make_float4(Tp.x * f.x * Le.x * k, Tp.y * f.y * Le.y * k, Tp.z * f.z * Le.z * k, 0.0f);
                            so = make_float4(pos.x, pos.y, pos.z, eps);
                            sd = make_float4(wi.x, wi.y, wi.z, dist * (1.0f - 1.0e-3f));
                            shadow = scv.x > 0.0f || scv.y > 0.0f || scv.z > 0.0f;
                        } else if (!mc && cos_l > 0.0f && cos_s > 0.0f && dist > 0.0f) {
                            const float pdf_l = inv_nl * dist2 / (tri_area(l0, l1, l2) * cos_l);
                            const float k = cos_s * kInvPi / (pdf_l * (float)(2u + cbase));
                            scv = make_float4(Tp.x * A.x * Le.x * k, Tp.y * A.y * Le.y * k, Tp.z * A.z * Le.z * k, 0.0f);
                            so = make_float4(pos.x, pos.y, pos.z, eps);
                            sd = make_float4(wi.x, wi.y, wi.z, dist * (1.0f - 1.0e-3f));
                            shadow = scv.x > 0.0f || scv.y > 0.0f || scv.z > 0.0f;
                        }
                    }
                    if (M > 0 && i + 2 <= Kmax) {  // s >= 2
                        for (uint32_t c = 0; c < C; c++) {
                            const uint32_t v = lvc_slot[vbase + min((uint32_t)(rng_u01(seed, key, vdim(b, 6) +
                                                                                         520u * (c + 1)) * (float)M),
                                                                    M - 1)];
                            const float4 vp4 = lvc_pos[v];
                            const uint32_t s = (uint32_t)vp4.w;
                            if (s + i > Kmax) continue;
                            const float4 vn4 = lvc_nrm[v];
                            const float3 dv = sub(xyz(vp4), pos);
                            const float dist2 = dot3(dv, dv), dist = sqrtf(dist2);
                            if (!(dist > 0.0f)) continue;
                            const float3 dir = mul(dv, 1.0f / dist);
                            const float cos_c = dot3(nrm, dir), cos_v = -dot3(xyz(vn4), dir);
                            const uint32_t vmat = __float_as_uint(vn4.w);
                            const MaterialDev* mv = lvc_wi ? layered_material(sc, vmat) : nullptr;
                            const float4 Av = sc.albedo[vmat];
                            const float4 bv = lvc_beta[v];
                            float4 cv;
                            if (mc || mv) {
                                float3 fc = f3(0.0f, 0.0f, 0.0f), fv = f3(0.0f, 0.0f, 0.0f);
                                if (mc) fc = material_f(*mc, ng, wo, dir, wo_l, to_local(frc, dir));
                                else if (cos_c > 0.0f) fc = f3(A.x * kInvPi, A.y * kInvPi, A.z * kInvPi);
                                if (mv) {
                                    const float4 w4 = lvc_wi[v];
                                    const float3 ngv = mul(xyz(vn4), w4.w), wiv = xyz(w4), wov = mul(dir, -1.0f);
                                    const Frame frv = frame_from_z(ngv);
                                    fv = material_f(*mv, ngv, wov, wiv, to_local(frv, wov), to_local(frv, wiv));
                                } else if (cos_v > 0.0f) {
                                    fv = f3(Av.x * kInvPi, Av.y * kInvPi, Av.z * kInvPi);
                                }
                                const float g = fabsf(cos_c) * fabsf(cos_v) / dist2 * ((float)M / n_light_paths) /
                                                ((2.0f + (float)cbase + bv.w) * (float)C);
                                cv = make_float4(Tp.x * fc.x * fv.x * bv.x * g, Tp.y * fc.y * fv.y * bv.y * g,
                                                 Tp.z * fc.z * fv.z * bv.z * g, 0.0f);
                            } else {
                                if (!(cos_c > 0.0f && cos_v > 0.0f)) continue;
                                const float g = cos_c * cos_v / dist2 * kInvPi * kInvPi * ((float)M / n_light_paths) /
                                                ((2.0f + (float)cbase + bv.w) * (float)C);
                                cv = make_float4(Tp.x * A.x * Av.x * bv.x * g, Tp.y * A.y * Av.y * bv.y * g,
                                                 Tp.z * A.z * Av.z * bv.z * g, 0.0f);
                            }
                            if (!(cv.x > 0.0f || cv.y > 0.0f || cv.z > 0.0f)) continue;
                            cc[(size_t)path * C + c] = cv;
                            cro[c] = make_float4(pos.x, pos.y, pos.z, eps);
                            crd[c] = make_float4(dir.x, dir.y, dir.z, dist * (1.0f - 1.0e-3f));
                            conn[c] = true;
                        }
                    }
                    if (i < Kmax && mc) {
                        float3 wi;
                        float pdf;
                        bool spec;
                        const float3 f = material_sample(*mc, frc, ng, wo, rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                                         rng_u01(seed, key, vdim(b, kDimBsdfV)),
                                                         rng_u01(seed, key, vdim(b, kDimBsdfC)), wi, pdf, spec);
                        if (pdf > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) {
                            const float k = fabsf(dot3(wi, ng)) / pdf;
                            Tp.x *= f.x * k; Tp.y *= f.y * k; Tp.z *= f.z * k;
                            Tp.w = __uint_as_float(bd_advance(cst, !spec));
                            cont = isfinite(Tp.x) && isfinite(Tp.y) && isfinite(Tp.z) &&
                                   (Tp.x > 0.0f || Tp.y > 0.0f || Tp.z > 0.0f);
                            if (cont && b >= rr_start) {
                                const float q = fminf(rr_prob, luminance(xyz(Tp)));
                                if (!(rng_u01(seed, key, vdim(b, kDimRR)) < q)) cont = false;
                                else { Tp.x /= q; Tp.y /= q; Tp.z /= q; }
                            }
                            if (cont) {
                                T[path] = Tp;
                                new_o = make_float4(pos.x, pos.y, pos.z, eps);
                                new_d = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    } else if (i < Kmax) {
                        const float3 loc = cosine_hemisphere(rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                                             rng_u01(seed, key, vdim(b, kDimBsdfV)));
                        if (loc.z > 0.0f) {
                            const float3 wi = normalize3(to_world(frame_from_z(nrm), loc));
                            Tp.x *= A.x; Tp.y *= A.y; Tp.z *= A.z;
                            Tp.w = __uint_as_float(bd_advance(cst, true));
                            cont = Tp.x > 0.0f || Tp.y > 0.0f || Tp.z > 0.0f;
                            if (cont && b >= rr_start) {
                                const float q = fminf(rr_prob, luminance(xyz(Tp)));
                                if (!(rng_u01(seed, key, vdim(b, kDimRR)) < q)) cont = false;
                                else { Tp.x /= q; Tp.y /= q; Tp.z /= q; }
                            }
                            if (cont) {
                                T[path] = Tp;
                                new_o = make_float4(pos.x, pos.y, pos.z, eps);
                                new_d = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    }
                }
            }
        }
        const uint32_t s_slot = warp_append(&wc->n_shadow, shadow);
        if (shadow) {
            srays[2 * (size_t)path] = so;
            srays[2 * (size_t)path + 1] = sd;
            sc_out[path] = scv;
            qs[s_slot] = path;
        }
        for (uint32_t c = 0; c < C; c++) {
            const uint32_t c_slot = warp_append(&wc->n_conn, conn[c]);
            if (conn[c]) {
                const size_t cs = (size_t)path * C + c;
                cray[2 * cs] = cro[c];
                cray[2 * cs + 1] = crd[c];
                cq[c_slot] = (uint32_t)cs;
            }
        }
        const uint32_t e_slot = warp_append(&wc->n_ext[cur ^ 1u], cont);
        if (cont) {
            rays[2 * (size_t)path] = new_o;
            rays[2 * (size_t)path + 1] = new_d;
            q_out[e_slot] = path;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&wc->stats[i == 1 ? 0 : 1], (unsigned long long)n);
}

// ---- BDPT: the reference's own estimator (integrators/integrator_bdpt_lvc_sk.cu) ---------
// Same wavefront stages and buffers as above; only the estimator differs
// (rb2_bdpt_lvc_params, RB2_BDPT_ESTIMATOR_REFERENCE).

// The reference's triangle area (compute_area, core/primitives.h:273-276) is
// 0.5 * length(compute_normal(...)), and compute_normal is normalized: every
// triangle's area is 0.5 in its light pdfs.
constexpr float kRefTriArea = 0.5f;
// Random dimensions of the BSDF half of the reference estimator's NEE (the
// same at every vertex, as its re-seeded NEE generator draws them).
constexpr uint32_t kDimNeeBsdf = 8000;

// intersect_ray_triangle (core/primitives.cu:51-70): Moller-Trumbore without a
// distance check, determinant threshold 1e-6; returns t.
__device__ __forceinline__ bool ref_intersect(float3 o, float3 d, float3 v0, float3 v1, float3 v2, float& t)
{
    const float3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    const float3 pv = cross3(d, e2);
    const float det = dot3(e1, pv);
    if (det < 1.0e-6f && det > -1.0e-6f) return false;
    const float inv = 1.0f / det;
    const float3 tv = sub(o, v0);
    const float u = dot3(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 qv = cross3(tv, e1);
    const float v = dot3(d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot3(e2, qv) * inv;
    return true;
}

// Light subpath start as DiffuseAreaLight::Le computes it (core/lights.cu:63-69,
// integrator_bdpt_lvc_sk.cu:61-83): uniform emissive triangle, uniform point,
// a direction uniform over the hemisphere about world +z (uniform_sample_hemisphere,
// core/montecarlo.cu:115-122) negated whenever its dot product with the light
// normal is nonzero; contribution Le / pdf, pdf = (1 / area) (1 / 2 pi) / |cos|,
// Le only toward the light's front, no factor for the triangle choice.
__global__ void k_bd_light_init_ref(SceneView sc, uint64_t seed, uint64_t key0, uint32_t n_paths, float4* lray,
                                    float4* lbeta, uint32_t* lq0, WaveCountersDev* wc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wc->n_ext[0] = sc.n_lights ? n_paths : 0u;
    if (!sc.n_lights) return;
    const uint64_t ls = seed ^ kLightSalt;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_paths; p += gridDim.x * blockDim.x) {
        const uint64_t key = key0 + p;
        uint32_t j = min((uint32_t)(rng_u01(ls, key, 0) * (float)sc.n_lights), sc.n_lights - 1);
        const uint4 lt = sc.tris[sc.lights[j]];
        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
        const float3 y0 = sample_triangle(l0, l1, l2, rng_u01(ls, key, 1), rng_u01(ls, key, 2));
        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
        const float hz = rng_u01(ls, key, 3);
        const float hr = sqrtf(fmaxf(0.0f, 1.0f - hz * hz)), phi = 6.283185307179586f * rng_u01(ls, key, 4);
        float3 dir = f3(hr * cosf(phi), hr * sinf(phi), hz);
        if (dot3(dir, ln) != 0.0f) dir = mul(dir, -1.0f);
        const float c = dot3(ln, dir);
        const float4 Le = sc.emission[lt.w];
        // pdf uses compute_area, which is 0.5 for every triangle (core/primitives.h:273-276:
        // half the length of the already normalized normal).
        const float k = c > 0.0f ? kRefTriArea * 6.283185307179586f * c : 0.0f;
        lbeta[p] = make_float4(Le.x * k, Le.y * k, Le.z * k, 0.0f);
        lray[2 * (size_t)p] = make_float4(y0.x, y0.y, y0.z, kLightRayTmin);
        lray[2 * (size_t)p + 1] = make_float4(dir.x, dir.y, dir.z, 3.402823466e+38f);
        lq0[p] = p;
    }
}

// Light vertex d (integrator_bdpt_lvc_sk.cu:93-166): every surface hit is
// stored, whatever its material and contribution (an emitter's BSDF is black:
// it is stored with zero contribution and ends the subpath); the subpath goes
// on with the sampled f |cos| / pdf and Russian roulette at every bounce,
// continue probability min(1, luminance), until its contribution is black.
__global__ void k_bd_light_shade_ref(SceneView sc, uint64_t seed, uint64_t key0, uint32_t d, uint32_t Dl,
                                     const uint32_t* q_in, uint32_t* q_out, float4* lray, const int4* lhit,
                                     float4* lbeta, float4* s_pos, float4* s_nrm, float4* s_beta, float4* s_wi,
                                     uint8_t* s_valid, WaveCountersDev* wc, uint32_t cur)
{
    const uint32_t n = wc->n_ext[cur];
    const uint64_t ls = seed ^ kLightSalt;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool cont = false;
        uint32_t path = 0;
        float4 no, nd;
        if (i < n) {
            path = q_in[i];
            const int4 h = lhit[path];
            if (h.x >= 0) {
                const float4 o4 = lray[2 * (size_t)path], d4 = lray[2 * (size_t)path + 1];
                const float t = __int_as_float(h.y);
                const float3 dd = xyz(d4);
                const float3 pos = f3(fmaf(dd.x, t, o4.x), fmaf(dd.y, t, o4.y), fmaf(dd.z, t, o4.z));
                const uint4 tri = sc.tris[h.x];
                const float4 E = sc.emission[tri.w];
                const bool emitter = E.x > 0.0f || E.y > 0.0f || E.z > 0.0f;
                const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
                const float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
                const float3 wo = mul(dd, -1.0f);
                const float3 nrm = dot3(ng, wo) < 0.0f ? mul(ng, -1.0f) : ng;
                float4 beta = lbeta[path];
                const size_t slot = (size_t)path * Dl + (d - 1);
                s_pos[slot] = make_float4(pos.x, pos.y, pos.z, (float)(d + 1));
                s_nrm[slot] = make_float4(nrm.x, nrm.y, nrm.z, __uint_as_float(tri.w));
                s_beta[slot] = emitter ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : make_float4(beta.x, beta.y, beta.z, 0.0f);
                s_valid[slot] = 1;
                if (s_wi) s_wi[slot] = make_float4(wo.x, wo.y, wo.z, dot3(ng, nrm) < 0.0f ? -1.0f : 1.0f);
                if (!emitter && d < Dl) {
                    const uint64_t key = key0 + path;
                    const MaterialDev* lm = layered_material(sc, tri.w);
                    float3 fac = f3(0.0f, 0.0f, 0.0f), wi = f3(0.0f, 0.0f, 0.0f);
                    bool ok = false;
                    if (lm) {
                        float pdf, eta_io;
                        bool spec;
                        const float3 f = material_sample(*lm, frame_from_z(ng), ng, wo, rng_u01(ls, key, 8 + 8 * d),
                                                         rng_u01(ls, key, 9 + 8 * d), rng_u01(ls, key, 11 + 8 * d), wi,
                                                         pdf, spec, &eta_io);
                        if (pdf > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) {
                            const float k = fabsf(dot3(wi, ng)) / pdf;
                            fac = f3(f.x * k, f.y * k, f.z * k);
                            ok = isfinite(fac.x) && isfinite(fac.y) && isfinite(fac.z);
                        }
                    } else {
                        const float3 loc = cosine_hemisphere(rng_u01(ls, key, 8 + 8 * d), rng_u01(ls, key, 9 + 8 * d));
                        if (loc.z > 0.0f) {
                            wi = normalize3(to_world(frame_from_z(nrm), loc));
                            fac = xyz(sc.albedo[tri.w]);
                            ok = true;
                        }
                    }
                    if (ok) {
                        const float q = fminf(1.0f, luminance(fac));
                        cont = q > 0.0f && rng_u01(ls, key, 10 + 8 * d) < q;
                        if (cont) {
                            beta.x *= fac.x / q; beta.y *= fac.y / q; beta.z *= fac.z / q;
                            cont = beta.x > 0.0f || beta.y > 0.0f || beta.z > 0.0f;
                        }
                        if (cont) {
                            lbeta[path] = beta;
                            no = make_float4(pos.x, pos.y, pos.z, 1.0e-3f * t);
                            nd = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                        }
                    }
                }
            }
        }
        const uint32_t slot_out = warp_append(&wc->n_ext[cur ^ 1u], cont);
        if (cont) {
            lray[2 * (size_t)path] = no;
            lray[2 * (size_t)path + 1] = nd;
            q_out[slot_out] = path;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&wc->stats[4], (unsigned long long)n);
}

// Camera vertex i = bounce + 1 (integrator_bdpt_lvc_sk.cu:186-434): emission
// on the first vertex or after a specular bounce (full weight, ends the path),
// next-event estimation at full weight with the draws of the first vertex at
// every vertex (the reference re-seeds its NEE generator each bounce), C
// connections to uniformly chosen cached vertices of this iteration, each
// weighted 1 / (i + depth of the cached vertex) with no cache-size factor,
// then the BSDF continuation and Russian roulette from bounce rr_start + 1
// dividing survivors by 1 - q.  The first `lvc_cap` cached vertices of the
// iteration (in (path, depth) order) are the cache.
__global__ void k_bd_cam_shade_ref(SceneView sc, uint64_t seed, uint32_t npix, uint32_t it0, uint32_t i, uint32_t Kc,
                                   uint32_t C, uint32_t Cs, uint32_t rr_start, float rr_prob, uint32_t lvc_cap,
                                   const uint32_t* q_in,
                                   uint32_t* q_out, float4* rays, const int4* hits, float4* T, float4* L, float4* srays,
                                   float4* sc_out, uint32_t* qs, float4* cray, float4* cc, uint32_t* cq,
                                   const float4* lvc_pos, const float4* lvc_nrm, const float4* lvc_beta,
                                   const float4* lvc_wi, const uint32_t* lvc_slot, const uint32_t* lvc_off,
                                   WaveCountersDev* wc, uint32_t cur)
{
    const uint32_t n = wc->n_ext[cur];
    const float inv_nl = sc.n_lights ? 1.0f / (float)sc.n_lights : 0.0f;
    const uint32_t b = i - 1;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t qi = base + threadIdx.x;
        bool cont = false, shadow = false;
        // Slots 0..C-1: cache connections; slot C: the BSDF half of NEE (an
        // occlusion segment to the light point it hits, same reduction).
        bool conn[kMaxConnections + 1];
        float4 cro[kMaxConnections + 1], crd[kMaxConnections + 1];
        for (uint32_t c = 0; c <= kMaxConnections; c++) conn[c] = false;
        uint32_t path = 0;
        float4 new_o, new_d, so, sd, scv;
        if (qi < n) {
            path = q_in[qi];
            for (uint32_t c = 0; c < Cs; c++) cc[(size_t)path * Cs + c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const int4 h = hits[path];
            if (h.x >= 0) {
                const uint64_t key = (uint64_t)it0 * npix + path;
                const uint32_t li = path / npix;
                const uint32_t vbase = lvc_off[li], M = min(lvc_off[li + 1] - vbase, lvc_cap);
                const float4 o4 = rays[2 * (size_t)path], d4 = rays[2 * (size_t)path + 1];
                const float t = __int_as_float(h.y);
                const float3 d = xyz(d4);
                const float3 pos = f3(fmaf(d.x, t, o4.x), fmaf(d.y, t, o4.y), fmaf(d.z, t, o4.z));
                const float eps = 1.0e-3f * t;
                const uint4 tri = sc.tris[h.x];
                const float3 v0 = xyz(sc.verts[tri.x]), v1 = xyz(sc.verts[tri.y]), v2 = xyz(sc.verts[tri.z]);
                const float3 ng = normalize3(cross3(sub(v1, v0), sub(v2, v0)));
                const float3 wo = mul(d, -1.0f);
                float4 Tp = T[path];
                const uint32_t cst = __float_as_uint(Tp.w);
                const float4 E = sc.emission[tri.w];
                if (E.x > 0.0f || E.y > 0.0f || E.z > 0.0f) {
                    // The camera counts as a specular vertex, so this covers bounce 0 too.
                    if (!bd_nonspec(cst) && dot3(ng, wo) > 0.0f) {
                        float4 Lp = L[path];
                        Lp.x += Tp.x * E.x; Lp.y += Tp.y * E.y; Lp.z += Tp.z * E.z;
                        L[path] = Lp;
                    }
                } else {
                    const float3 nrm = dot3(ng, wo) < 0.0f ? mul(ng, -1.0f) : ng;
                    const float4 A = sc.albedo[tri.w];
                    const MaterialDev* mc = layered_material(sc, tri.w);
                    const Frame frc = frame_from_z(ng);
                    const float3 wo_l = to_local(frc, wo);
                    if (sc.n_lights) {
                        // compute_direct_lighting's two halves for one uniformly chosen
                        // emissive triangle j (integrator_bdpt_lvc_sk.cu:233-327): a light
                        // sample and a BSDF sample, balance-heuristic weights from the
                        // reference's pdfs (area 0.5, no 1/n_lights), the sum times n_lights.
                        const float nl = (float)sc.n_lights;
                        uint32_t j = min((uint32_t)(rng_u01(seed, key, vdim(0, kDimLight)) * nl), sc.n_lights - 1);
                        const uint4 lt = sc.tris[sc.lights[j]];
                        const float3 l0 = xyz(sc.verts[lt.x]), l1 = xyz(sc.verts[lt.y]), l2 = xyz(sc.verts[lt.z]);
                        const float3 ln = normalize3(cross3(sub(l1, l0), sub(l2, l0)));
                        const float4 Le = sc.emission[lt.w];
                        {
                            const float3 lp = sample_triangle(l0, l1, l2, rng_u01(seed, key, vdim(0, kDimLightU)),
                                                              rng_u01(seed, key, vdim(0, kDimLightV)));
                            const float3 dv = sub(lp, pos);
                            const float dist2 = dot3(dv, dv), dist = sqrtf(dist2);
                            const float3 wi = mul(dv, 1.0f / dist);
                            const float cos_l = -dot3(ln, wi), cos_s = dot3(nrm, wi);
                            float3 f = f3(0.0f, 0.0f, 0.0f);
                            float pdf_b = 0.0f;
                            if (mc) {
                                const float3 wi_l = to_local(frc, wi);
                                f = material_f(*mc, ng, wo, wi, wo_l, wi_l);
                                pdf_b = material_pdf(*mc, wo_l, wi_l);
                            } else if (cos_s > 0.0f) {
                                f = f3(A.x * kInvPi, A.y * kInvPi, A.z * kInvPi);
                                pdf_b = cos_s * kInvPi;
                            }
                            if (cos_l > 0.0f && dist > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) {
                                const float pdf_l = dist2 / (kRefTriArea * cos_l);
                                const float k = fabsf(cos_s) * (pdf_l / (pdf_l + pdf_b)) / pdf_l * nl;
                                scv = make_float4(Tp.x * f.x * Le.x * k, Tp.y * f.y * Le.y * k, Tp.z * f.z * Le.z * k,
                                                  0.0f);
                                so = make_float4(pos.x, pos.y, pos.z, eps);
                                sd = make_float4(wi.x, wi.y, wi.z, dist * (1.0f - 1.0e-3f));
                                shadow = scv.x > 0.0f || scv.y > 0.0f || scv.z > 0.0f;
                            }
                        }
                        {
                            float3 wi = f3(0.0f, 0.0f, 0.0f), f = f3(0.0f, 0.0f, 0.0f);
                            float pdf_b = 0.0f;
                            if (mc) {
                                bool spec;
                                f = material_sample(*mc, frc, ng, wo, rng_u01(seed, key, kDimNeeBsdf),
                                                    rng_u01(seed, key, kDimNeeBsdf + 1),
                                                    rng_u01(seed, key, kDimNeeBsdf + 2), wi, pdf_b, spec);
                                if (spec) pdf_b = 0.0f;  // the reference samples the non-specular layers here
                            } else {
                                const float3 loc = cosine_hemisphere(rng_u01(seed, key, kDimNeeBsdf),
                                                                     rng_u01(seed, key, kDimNeeBsdf + 1));
                                if (loc.z > 0.0f) {
                                    wi = normalize3(to_world(frame_from_z(nrm), loc));
                                    f = f3(A.x * kInvPi, A.y * kInvPi, A.z * kInvPi);
                                    pdf_b = loc.z * kInvPi;
                                }
                            }
                            float th;
                            if (pdf_b > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f) &&
                                ref_intersect(pos, wi, l0, l1, l2, th) && th > eps) {
                                const float cth = dot3(ln, mul(wi, -1.0f));   // L(-wi): front side only
                                const float pdf_l = th * th / (kRefTriArea * fabsf(cth));
                                const float k = (cth > 0.0f ? 1.0f : 0.0f) * fabsf(dot3(wi, nrm)) *
                                                (pdf_b / (pdf_b + pdf_l)) / pdf_b * nl;
                                const float4 cv = make_float4(Tp.x * f.x * Le.x * k, Tp.y * f.y * Le.y * k,
                                                              Tp.z * f.z * Le.z * k, 0.0f);
                                if (cv.x > 0.0f || cv.y > 0.0f || cv.z > 0.0f) {
                                    // The reference counts it when the BSDF ray's closest hit is
                                    // triangle j: the segment up to it must be unoccluded.
                                    cc[(size_t)path * Cs + C] = cv;
                                    cro[C] = make_float4(pos.x, pos.y, pos.z, eps);
                                    crd[C] = make_float4(wi.x, wi.y, wi.z, th * (1.0f - 1.0e-3f));
                                    conn[C] = true;
                                }
                            }
                        }
                    }
                    if (M > 0) {
                        for (uint32_t c = 0; c < C; c++) {
                            const uint32_t v = lvc_slot[vbase + min((uint32_t)(rng_u01(seed, key, vdim(b, 6) +
                                                                                         520u * (c + 1)) * (float)M),
                                                                    M - 1)];
                            const float4 vp4 = lvc_pos[v];
                            const float depth = vp4.w - 1.0f;  // the reference's m_depth: 1 at the first hit
                            const float4 vn4 = lvc_nrm[v];
                            const float3 dv = sub(xyz(vp4), pos);
                            const float dist2 = dot3(dv, dv), dist = sqrtf(dist2);
                            if (!(dist > 0.0f)) continue;
                            const float3 dir = mul(dv, 1.0f / dist);
                            const float cos_c = dot3(nrm, dir), cos_v = -dot3(xyz(vn4), dir);
                            const uint32_t vmat = __float_as_uint(vn4.w);
                            const MaterialDev* mv = lvc_wi ? layered_material(sc, vmat) : nullptr;
                            const float4 Av = sc.albedo[vmat];
                            const float4 bv = lvc_beta[v];
                            float3 fc = f3(0.0f, 0.0f, 0.0f), fv = f3(0.0f, 0.0f, 0.0f);
                            if (mc) fc = material_f(*mc, ng, wo, dir, wo_l, to_local(frc, dir));
                            else if (cos_c > 0.0f) fc = f3(A.x * kInvPi, A.y * kInvPi, A.z * kInvPi);
                            if (mv) {
                                // material_f(lvc material, wo = toward the previous light vertex,
                                // wi = toward the camera vertex), as the reference orders them.
                                const float4 w4 = lvc_wi[v];
                                const float3 ngv = mul(xyz(vn4), w4.w), wov = xyz(w4), wiv = mul(dir, -1.0f);
                                const Frame frv = frame_from_z(ngv);
                                fv = material_f(*mv, ngv, wov, wiv, to_local(frv, wov), to_local(frv, wiv));
                            } else if (cos_v > 0.0f) {
                                fv = f3(Av.x * kInvPi, Av.y * kInvPi, Av.z * kInvPi);
                            }
                            const float g = fabsf(cos_c) * fabsf(cos_v) / dist2 / ((float)i + depth);
                            const float4 cv = make_float4(Tp.x * fc.x * fv.x * bv.x * g, Tp.y * fc.y * fv.y * bv.y * g,
                                                          Tp.z * fc.z * fv.z * bv.z * g, 0.0f);
                            if (!(cv.x > 0.0f || cv.y > 0.0f || cv.z > 0.0f)) continue;
                            cc[(size_t)path * Cs + c] = cv;
                            cro[c] = make_float4(pos.x, pos.y, pos.z, eps);
                            crd[c] = make_float4(dir.x, dir.y, dir.z, dist * (1.0f - 1.0e-3f));
                            conn[c] = true;
                        }
                    }
                    if (i < Kc) {
                        float3 wi = f3(0.0f, 0.0f, 0.0f);
                        bool ok = false, spec = false;
                        if (mc) {
                            float pdf;
                            const float3 f = material_sample(*mc, frc, ng, wo, rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                                             rng_u01(seed, key, vdim(b, kDimBsdfV)),
                                                             rng_u01(seed, key, vdim(b, kDimBsdfC)), wi, pdf, spec);
                            if (pdf > 0.0f && (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f)) {
                                const float k = fabsf(dot3(wi, ng)) / pdf;
                                Tp.x *= f.x * k; Tp.y *= f.y * k; Tp.z *= f.z * k;
                                ok = true;
                            }
                        } else {
                            const float3 loc = cosine_hemisphere(rng_u01(seed, key, vdim(b, kDimBsdfU)),
                                                                 rng_u01(seed, key, vdim(b, kDimBsdfV)));
                            if (loc.z > 0.0f) {
                                wi = normalize3(to_world(frame_from_z(nrm), loc));
                                Tp.x *= A.x; Tp.y *= A.y; Tp.z *= A.z;
                                ok = true;
                            }
                        }
                        if (ok) {
                            Tp.w = __uint_as_float(bd_advance(cst, !spec));
                            cont = isfinite(Tp.x) && isfinite(Tp.y) && isfinite(Tp.z) &&
                                   (Tp.x > 0.0f || Tp.y > 0.0f || Tp.z > 0.0f);
                            if (cont && b > rr_start) {
                                const float q = fminf(rr_prob, luminance(xyz(Tp)));
                                if (!(rng_u01(seed, key, vdim(b, kDimRR)) < q)) cont = false;
                                else { const float inv = 1.0f / (1.0f - q); Tp.x *= inv; Tp.y *= inv; Tp.z *= inv; }
                            }
                            if (cont) {
                                T[path] = Tp;
                                new_o = make_float4(pos.x, pos.y, pos.z, eps);
                                new_d = make_float4(wi.x, wi.y, wi.z, 3.402823466e+38f);
                            }
                        }
                    }
                }
            }
        }
        const uint32_t s_slot = warp_append(&wc->n_shadow, shadow);
        if (shadow) {
            srays[2 * (size_t)path] = so;
            srays[2 * (size_t)path + 1] = sd;
            sc_out[path] = scv;
            qs[s_slot] = path;
        }
        for (uint32_t c = 0; c < Cs; c++) {
            const uint32_t c_slot = warp_append(&wc->n_conn, conn[c]);
            if (conn[c]) {
                const size_t cs = (size_t)path * Cs + c;
                cray[2 * cs] = cro[c];
                cray[2 * cs + 1] = crd[c];
                cq[c_slot] = (uint32_t)cs;
            }
        }
        const uint32_t e_slot = warp_append(&wc->n_ext[cur ^ 1u], cont);
        if (cont) {
            rays[2 * (size_t)path] = new_o;
            rays[2 * (size_t)path + 1] = new_d;
            q_out[e_slot] = path;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&wc->stats[i == 1 ? 0 : 1], (unsigned long long)n);
}

__global__ void k_bd_stats(WaveCountersDev* wc)
{
    wc->stats[2] += wc->n_shadow;
    wc->stats[3] += wc->n_conn;
}

// Adds the surviving connection contributions of each shaded path, in
// connection order (deterministic).
__global__ void k_bd_conn_reduce(const uint32_t* q_in, const WaveCountersDev* wc, uint32_t cur, uint32_t C,
                                 const float4* cc, float4* L)
{
    const uint32_t n = wc->n_ext[cur];
    for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
        const uint32_t path = q_in[qi];
        float4 a = L[path];
        for (uint32_t c = 0; c < C; c++) {
            const float4 v = cc[(size_t)path * C + c];
            a.x += v.x; a.y += v.y; a.z += v.z;
        }
        L[path] = a;
    }
}

__global__ void k_pt_finalize(const float4* accum, uint32_t npix, float inv_spp, float* rgb)
{
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        const float4 a = accum[pix];
        rgb[3 * (size_t)pix + 0] = a.x * inv_spp;
        rgb[3 * (size_t)pix + 1] = a.y * inv_spp;
        rgb[3 * (size_t)pix + 2] = a.z * inv_spp;
    }
}

}  // namespace rb2dev

namespace {

template <int B, int R, int LAYOUT, class Src>
int launch_persistent_variant(const Src& src, uint64_t work, int sms, uint32_t threshold, uint32_t node_threshold,
                              unsigned int* status, cudaStream_t s)
{
    int per_sm = 0;
    RB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rb2dev::k_persistent<B, R, Src, LAYOUT>, B, 0),
             "occupancy");
    uint64_t blocks = (uint64_t)sms * (uint64_t)std::max(1, per_sm);
    blocks = std::min<uint64_t>(blocks, (work + B - 1) / B);
    blocks = std::max<uint64_t>(blocks, 1);
    rb2dev::k_persistent<B, R, Src, LAYOUT><<<(unsigned)blocks, B, 0, s>>>(src, threshold, node_threshold, status);
    RB2_CUDA(cudaGetLastError(), "persistent launch");
    return RB2_OK;
}

template <int LAYOUT, class Src>
int launch_persistent_shape(const Src& src, uint64_t work, const rb2_integrator* it, unsigned int* status, cudaStream_t s)
{
    const uint32_t th = it->tr_threshold;
    // Node-phase threshold: on the config-2/3 rooms 16 was the fastest for the
    // compressed layout (path tracer 307.5 ms vs 309.2 at 12 and 366.3 at 1;
    // BDPT 83.1 vs 86.5 and 104.3 ms); the binary layout keeps its default.
    const uint32_t nt = it->tr_node_threshold ? it->tr_node_threshold
                                              : (LAYOUT == rb2dev::kLayoutCw8 ? 16u : rb2dev::default_node_threshold(LAYOUT));
    const uint32_t regs = it->tr_regs ? it->tr_regs : (LAYOUT == rb2dev::kLayoutCw8 ? 64u : 48u);
    if (it->tr_block == 256)
        return regs == 48 ? launch_persistent_variant<256, 48, LAYOUT>(src, work, it->sms, th, nt, status, s)
                                 : launch_persistent_variant<256, 64, LAYOUT>(src, work, it->sms, th, nt, status, s);
    return regs == 48 ? launch_persistent_variant<128, 48, LAYOUT>(src, work, it->sms, th, nt, status, s)
                             : launch_persistent_variant<128, 64, LAYOUT>(src, work, it->sms, th, nt, status, s);
}

template <class Src>
int launch_persistent_layout(const Src& src, uint64_t work, const rb2_integrator* it, unsigned int* status, bool cw8,
                             cudaStream_t s)
{
    return cw8 ? launch_persistent_shape<rb2dev::kLayoutCw8>(src, work, it, status, s)
               : launch_persistent_shape<rb2dev::kLayoutBinary>(src, work, it, status, s);
}

// With timing on, each traversal launch is bracketed by an event pair.  The
// layout is the view's (the tracer's compressed 8-wide layout when it uses one).
template <class Src>
int launch_persistent(const Src& src, uint64_t work, rb2_integrator* it, const DeviceBvhView& bv, cudaStream_t s)
{
    unsigned int* status = bv.status;
    if (!it->timing) return launch_persistent_layout(src, work, it, status, bv.cw8, s);
    while (it->ev.size() < it->ev_used + 2) {
        cudaEvent_t e;
        RB2_CUDA(cudaEventCreate(&e), "timing event");
        it->ev.push_back(e);
    }
    RB2_CUDA(cudaEventRecord(it->ev[it->ev_used], s), "timing event");
    const int rc = launch_persistent_layout(src, work, it, status, bv.cw8, s);
    if (rc) return rc;
    RB2_CUDA(cudaEventRecord(it->ev[it->ev_used + 1], s), "timing event");
    it->ev_used += 2;
    return RB2_OK;
}

unsigned grid_for(uint64_t n, int sms) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 8)); }

}  // namespace

namespace rb2 {

int ensure_path_state(PathState& ps, uint64_t P)
{
    if (P <= ps.cap) return RB2_OK;
    rb2::dev_free(ps.T); rb2::dev_free(ps.L); rb2::dev_free(ps.ray); rb2::dev_free(ps.hit); rb2::dev_free(ps.sray); rb2::dev_free(ps.sc);
    rb2::dev_free(ps.q[0]); rb2::dev_free(ps.q[1]); rb2::dev_free(ps.qs);
    ps = PathState();
    cudaError_t e;
    if ((e = rb2::dev_malloc(&ps.T, P * 16)) != cudaSuccess || (e = rb2::dev_malloc(&ps.L, P * 16)) != cudaSuccess ||
        (e = rb2::dev_malloc(&ps.ray, P * 32)) != cudaSuccess || (e = rb2::dev_malloc(&ps.hit, P * 16)) != cudaSuccess ||
        (e = rb2::dev_malloc(&ps.sray, P * 32)) != cudaSuccess || (e = rb2::dev_malloc(&ps.sc, P * 16)) != cudaSuccess ||
        (e = rb2::dev_malloc(&ps.q[0], P * 4)) != cudaSuccess || (e = rb2::dev_malloc(&ps.q[1], P * 4)) != cudaSuccess ||
        (e = rb2::dev_malloc(&ps.qs, P * 4)) != cudaSuccess)
        return fail(RB2_ENOMEM, std::string("path state: ") + cudaGetErrorString(e));
    ps.cap = P;
    return RB2_OK;
}

int ensure_bdpt_state(BdptState& bd, uint64_t n_paths, uint64_t n_slots, uint64_t n_conn)
{
    cudaError_t e = cudaSuccess;
    if (!bd.lvc_off && (e = rb2::dev_malloc(&bd.lvc_off, (kMaxBdptWave + 1) * sizeof(uint32_t))) != cudaSuccess)
        return fail(RB2_ENOMEM, std::string("cache offsets: ") + cudaGetErrorString(e));
    if (n_paths > bd.cap_paths) {
        for (void* p : {(void*)bd.lray, (void*)bd.lbeta, (void*)bd.lhit, (void*)bd.lq[0], (void*)bd.lq[1]}) rb2::dev_free(p);
        bd.lray = bd.lbeta = nullptr; bd.lhit = nullptr; bd.lq[0] = bd.lq[1] = nullptr; bd.cap_paths = 0;
        if ((e = rb2::dev_malloc(&bd.lray, n_paths * 32)) != cudaSuccess || (e = rb2::dev_malloc(&bd.lbeta, n_paths * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.lhit, n_paths * 16)) != cudaSuccess || (e = rb2::dev_malloc(&bd.lq[0], n_paths * 4)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.lq[1], n_paths * 4)) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("light paths: ") + cudaGetErrorString(e));
        bd.cap_paths = n_paths;
    }
    if (n_slots > bd.cap_slots) {
        for (void* p : {(void*)bd.s_pos, (void*)bd.s_nrm, (void*)bd.s_beta, (void*)bd.s_wi, (void*)bd.s_valid,
                        (void*)bd.d_slot, (void*)bd.block_sums})
            rb2::dev_free(p);
        bd.s_pos = bd.s_nrm = bd.s_beta = bd.s_wi = nullptr;
        bd.s_valid = nullptr; bd.d_slot = nullptr; bd.block_sums = nullptr; bd.cap_slots = 0;
        const uint64_t nb = (n_slots + rb2dev::kScanChunk - 1) / rb2dev::kScanChunk;
        if ((e = rb2::dev_malloc(&bd.s_pos, n_slots * 16)) != cudaSuccess || (e = rb2::dev_malloc(&bd.s_nrm, n_slots * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.s_beta, n_slots * 16)) != cudaSuccess || (e = rb2::dev_malloc(&bd.s_valid, n_slots)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.d_slot, n_slots * 4)) != cudaSuccess || (e = rb2::dev_malloc(&bd.s_wi, n_slots * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.block_sums, nb * 4)) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("light vertex cache: ") + cudaGetErrorString(e));
        bd.cap_slots = n_slots;
    }
    if (n_conn > bd.cap_conn) {
        for (void* p : {(void*)bd.cray, (void*)bd.cc, (void*)bd.cq}) rb2::dev_free(p);
        bd.cray = bd.cc = nullptr; bd.cq = nullptr; bd.cap_conn = 0;
        if ((e = rb2::dev_malloc(&bd.cray, n_conn * 32)) != cudaSuccess || (e = rb2::dev_malloc(&bd.cc, n_conn * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&bd.cq, n_conn * 4)) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("connection rays: ") + cudaGetErrorString(e));
        bd.cap_conn = n_conn;
    }
    return RB2_OK;
}

uint64_t pt_paths_in_flight(uint64_t npix, uint32_t spp, uint32_t spp_per_wave, uint64_t auto_paths)
{
    uint32_t spw = spp_per_wave ? spp_per_wave
                                : (uint32_t)std::max<uint64_t>(1, auto_paths / std::max<uint64_t>(1, npix));
    spw = std::min(spw, std::max<uint32_t>(1, spp));
    return npix * spw;
}

int integrator_reserve_pt(rb2_integrator* it, uint64_t paths, uint64_t npix)
{
    int rc;
    if ((rc = ensure_path_state(it->ps, paths))) return rc;
    if ((rc = grow(it->d_accum, it->cap_accum, npix))) return rc;
    if (!it->d_wave) RB2_CUDA(rb2::dev_malloc(&it->d_wave, sizeof(WaveCounters)), "wave counters");
    return RB2_OK;
}

}  // namespace rb2

extern "C" {

int rb2_scene_create(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, const uint32_t* tri_material,
                     uint32_t n_materials, const float* albedo_rgb, const float* emission_rgb, rb2_scene_dev** out)
{
    if (!out || (nv && !v_xyz) || (ntri && !idx3)) return fail(RB2_EINVAL, "null scene argument");
    *out = nullptr;
    for (uint64_t i = 0; i < 3ull * ntri; i++)
        if (idx3[i] >= nv) return fail(RB2_EINVAL, "scene triangle index out of range");
    const uint32_t nm = std::max<uint32_t>(1, n_materials);
    if (tri_material)
        for (uint32_t i = 0; i < ntri; i++)
            if (tri_material[i] >= nm) return fail(RB2_EINVAL, "material id out of range");
    std::vector<float4> v(std::max<uint32_t>(1, nv));
    for (uint32_t i = 0; i < nv; i++) v[i] = make_float4(v_xyz[3 * i], v_xyz[3 * i + 1], v_xyz[3 * i + 2], 0.0f);
    std::vector<uint4> t(std::max<uint32_t>(1, ntri));
    std::vector<float4> alb(nm), emi(nm);
    for (uint32_t m = 0; m < nm; m++) {
        alb[m] = albedo_rgb ? make_float4(albedo_rgb[3 * m], albedo_rgb[3 * m + 1], albedo_rgb[3 * m + 2], 0.0f)
                            : make_float4(0.5f, 0.5f, 0.5f, 0.0f);
        emi[m] = emission_rgb ? make_float4(emission_rgb[3 * m], emission_rgb[3 * m + 1], emission_rgb[3 * m + 2], 0.0f)
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    std::vector<uint32_t> lights;
    for (uint32_t i = 0; i < ntri; i++) {
        uint32_t m = tri_material ? tri_material[i] : 0;
        t[i] = make_uint4(idx3[3 * i], idx3[3 * i + 1], idx3[3 * i + 2], m);
        const float4& e = emi[m];
        if (e.x > 0.0f || e.y > 0.0f || e.z > 0.0f) lights.push_back(i);  // core/scene.cpp:105-113
    }
    std::unique_ptr<rb2_scene_dev> s(new rb2_scene_dev());
    s->nv = nv; s->ntri = ntri; s->n_mat = nm; s->n_lights = (uint32_t)lights.size();
    if (lights.empty()) lights.push_back(0);
    cudaError_t e;
    if ((e = rb2::dev_malloc(&s->d_verts, v.size() * sizeof(float4))) != cudaSuccess ||
        (e = rb2::dev_malloc(&s->d_tris, t.size() * sizeof(uint4))) != cudaSuccess ||
        (e = rb2::dev_malloc(&s->d_albedo, nm * sizeof(float4))) != cudaSuccess ||
        (e = rb2::dev_malloc(&s->d_emission, nm * sizeof(float4))) != cudaSuccess ||
        (e = rb2::dev_malloc(&s->d_lights, lights.size() * sizeof(uint32_t))) != cudaSuccess) {
        rb2::dev_free(s->d_verts); rb2::dev_free(s->d_tris); rb2::dev_free(s->d_albedo); rb2::dev_free(s->d_emission); rb2::dev_free(s->d_lights);
        return fail(RB2_ENOMEM, std::string("scene allocation: ") + cudaGetErrorString(e));
    }
    RB2_CUDA(cudaMemcpy(s->d_verts, v.data(), v.size() * sizeof(float4), cudaMemcpyHostToDevice), "scene upload");
    RB2_CUDA(cudaMemcpy(s->d_tris, t.data(), t.size() * sizeof(uint4), cudaMemcpyHostToDevice), "scene upload");
    RB2_CUDA(cudaMemcpy(s->d_albedo, alb.data(), nm * sizeof(float4), cudaMemcpyHostToDevice), "scene upload");
    RB2_CUDA(cudaMemcpy(s->d_emission, emi.data(), nm * sizeof(float4), cudaMemcpyHostToDevice), "scene upload");
    RB2_CUDA(cudaMemcpy(s->d_lights, lights.data(), lights.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "scene upload");
    s->bytes = v.size() * 16 + t.size() * 16 + nm * 32 + lights.size() * 4;
    *out = s.release();
    return RB2_OK;
}

int rb2_scene_destroy(rb2_scene_dev* s)
{
    if (!s) return RB2_OK;
    rb2::dev_free(s->d_verts); rb2::dev_free(s->d_tris); rb2::dev_free(s->d_albedo); rb2::dev_free(s->d_emission); rb2::dev_free(s->d_lights);
    rb2::dev_free(s->d_mats);
    delete s;
    return RB2_OK;
}

int rb2_scene_device_bytes(const rb2_scene_dev* s, uint64_t* bytes)
{
    if (!s || !bytes) return fail(RB2_EINVAL, "null argument");
    *bytes = s->bytes;
    return RB2_OK;
}

int rb2_integrator_create(rb2_tracer* tracer, const rb2_scene_dev* scene, rb2_integrator** out)
{
    if (!tracer || !scene || !out) return fail(RB2_EINVAL, "null argument");
    *out = nullptr;
    std::unique_ptr<rb2_integrator> it(new rb2_integrator());
    it->tracer = tracer;
    it->scene = scene;
    int dev = 0;
    RB2_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    RB2_CUDA(cudaDeviceGetAttribute(&it->sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    RB2_CUDA(rb2::dev_malloc(&it->d_counters, 16 * sizeof(unsigned long long)), "integrator counters");
    *out = it.release();
    return RB2_OK;
}

int rb2_integrator_destroy(rb2_integrator* it)
{
    if (!it) return RB2_OK;
    rb2::dev_free(it->d_rays); rb2::dev_free(it->d_hits); rb2::dev_free(it->d_count); rb2::dev_free(it->d_counters);
    rb2::dev_free(it->d_accum); rb2::dev_free(it->d_wave); rb2::dev_free(it->d_film_xy);
    for (cudaEvent_t e : it->ev) cudaEventDestroy(e);
    PathState& ps = it->ps;
    rb2::dev_free(ps.T); rb2::dev_free(ps.L); rb2::dev_free(ps.ray); rb2::dev_free(ps.hit); rb2::dev_free(ps.sray); rb2::dev_free(ps.sc);
    rb2::dev_free(ps.q[0]); rb2::dev_free(ps.q[1]); rb2::dev_free(ps.qs);
    BdptState& bd = it->bd;
    for (void* p : {(void*)bd.lray, (void*)bd.lbeta, (void*)bd.lhit, (void*)bd.lq[0], (void*)bd.lq[1], (void*)bd.s_pos,
                    (void*)bd.s_nrm, (void*)bd.s_beta, (void*)bd.s_wi, (void*)bd.s_valid, (void*)bd.d_slot,
                    (void*)bd.block_sums, (void*)bd.cray,
                    (void*)bd.cc, (void*)bd.cq, (void*)bd.lvc_off})
        rb2::dev_free(p);
    delete it;
    return RB2_OK;
}

int rb2_integrator_set_launch(rb2_integrator* it, const rb2_launch_config* cfg)
{
    if (!it || !cfg) return fail(RB2_EINVAL, "null argument");
    if (cfg->block_threads && cfg->block_threads != 128 && cfg->block_threads != 256)
        return fail(RB2_ENOTSUP, "integrator traversal block_threads must be 128 or 256");
    if (cfg->regs && cfg->regs != 64 && cfg->regs != 48) return fail(RB2_ENOTSUP, "integrator regs must be 64 or 48");
    if (cfg->fetch_threshold > 32) return fail(RB2_EINVAL, "fetch_threshold must be <= 32");
    if (cfg->node_threshold > 32) return fail(RB2_EINVAL, "node_threshold must be <= 32");
    it->tr_block = cfg->block_threads ? cfg->block_threads : 128;
    it->tr_regs = cfg->regs;
    it->tr_threshold = cfg->fetch_threshold ? cfg->fetch_threshold : 24;
    it->tr_node_threshold = cfg->node_threshold;
    return RB2_OK;
}

int rb2_integrator_device_bytes(const rb2_integrator* it, uint64_t* bytes)
{
    if (!it || !bytes) return fail(RB2_EINVAL, "null argument");
    *bytes = it->bytes();
    return RB2_OK;
}

int rb2_render_ao(rb2_integrator* it, const rb2_camera* cam, const rb2_ao_params* p, float* d_ao, void* stream)
{
    rb2::Range nvtx_range("rb2_render_ao");
    if (!it || !cam || !p || !d_ao) return fail(RB2_EINVAL, "null argument");
    it->ev_used = 0;
    if (p->samples == 0 || !(p->radius > 0.0f)) return fail(RB2_EINVAL, "AO needs samples > 0 and radius > 0");
    if (p->compat & ~(uint32_t)RB2_COMPAT_AO_DIRECTION) return fail(RB2_EINVAL, "AO compat flags: RB2_COMPAT_AO_DIRECTION only");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t npix = (uint64_t)cam->width * cam->height;
    if (npix > 0xFFFFFFFFull) return fail(RB2_EINVAL, "image too large");
    int rc;
    if ((rc = grow(it->d_rays, it->cap_rays, 2 * npix)) || (rc = grow(it->d_hits, it->cap_hits, npix)) ||
        (rc = grow(it->d_count, it->cap_count, npix)))
        return rc;
    // 1. Primary rays through pixel centres, 2. closest hit (IntegratorAO::compute, integrator_ao.cu:92-101).
    if ((rc = rb2_camera_rays(cam, 1, 0, 0, reinterpret_cast<float*>(it->d_rays), stream))) return rc;
    if (it->timing) {
        while (it->ev.size() < it->ev_used + 2) {
            cudaEvent_t e;
            RB2_CUDA(cudaEventCreate(&e), "timing event");
            it->ev.push_back(e);
        }
        RB2_CUDA(cudaEventRecord(it->ev[it->ev_used], s), "timing event");
    }
    // Camera rays from beyond the compressed layout's origin bound go through the binary buffer.
    if (!cw8_origin_ok(it->tracer, cam->eye)) {
        if ((rc = trace_binary(it->tracer, reinterpret_cast<const float*>(it->d_rays), npix, 0, it->d_hits, s)))
            return rc;
    } else if ((rc = rb2_trace(it->tracer, reinterpret_cast<const float*>(it->d_rays), (uint32_t)npix, 0, nullptr,
                        reinterpret_cast<rb2_hit*>(it->d_hits), stream)))
        return rc;
    if (it->timing) {
        RB2_CUDA(cudaEventRecord(it->ev[it->ev_used + 1], s), "timing event");
        it->ev_used += 2;
    }
    // 3. AO rays generated and traced in one persistent launch, unoccluded counts per pixel.
    RB2_CUDA(cudaMemsetAsync(it->d_count, 0, npix * sizeof(uint32_t), s), "AO count reset");
    RB2_CUDA(cudaMemsetAsync(it->d_counters, 0, sizeof(unsigned long long), s), "queue reset");
    const DeviceBvhView bv = device_bvh(it->tracer, true);
    rb2dev::AoSource src;
    src.nodes = static_cast<const float4*>(bv.nodes);
    src.woop = static_cast<const float4*>(bv.woop);
    src.triidx = bv.triidx;
    src.prim_rays = it->d_rays;
    src.hits = it->d_hits;
    src.verts = it->scene->d_verts;
    src.tris = it->scene->d_tris;
    src.counts = it->d_count;
    src.counter = it->d_counters;
    src.n_slots = npix * p->samples;
    src.samples = p->samples;
    src.radius = p->radius;
    src.seed = p->seed;
    src.compat = p->compat;
    if ((rc = launch_persistent(src, src.n_slots, it, bv, s))) return rc;
    // 4. AO = unoccluded fraction (misses contribute 0, integrator_ao.cu:56-84).
    rb2dev::k_ao_finalize<<<grid_for(npix, it->sms), 256, 0, s>>>(it->d_hits, it->d_count, (uint32_t)npix, p->samples, d_ao);
    RB2_CUDA(cudaGetLastError(), "AO finalize");
    return RB2_OK;
}

namespace {

// The path tracer over samples [first_sample, first_sample + spp) of every
// pixel, added to `accum` (per pixel: r, g, b sums, and the filter weight sum
// in w when a film filter is set), which is zeroed first when `reset`; then,
// when d_rgb is given, the mean over the first_sample + spp samples summed so
// far.  Every random number is keyed by the sample's global index and the sums
// run in sample order, so unfiltered sums do not depend on how the samples are
// split into calls or waves.
int render_pt(rb2_integrator* it, const rb2_camera* cam, const rb2_pt_params* p, uint32_t first_sample, float4* accum,
              bool reset, float* d_rgb, void* stream)
{
    rb2::Range nvtx_range("rb2_render_pt");
    it->ev_used = 0;
    if (p->spp == 0) return fail(RB2_EINVAL, "spp must be > 0");
    if (p->max_depth > 64) return fail(RB2_EINVAL, "max_depth must be <= 64");
    if (p->compat & ~(uint32_t)(RB2_COMPAT_RR_DIVISOR | RB2_COMPAT_NEE_RESEED))
        return fail(RB2_EINVAL, "PT compat flags: RB2_COMPAT_RR_DIVISOR and RB2_COMPAT_NEE_RESEED only");
    if ((p->compat & RB2_COMPAT_RR_DIVISOR) && !(p->rr_prob < 1.0f))
        return fail(RB2_EINVAL, "RB2_COMPAT_RR_DIVISOR divides by 1 - q: rr_prob must be < 1");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t npix = (uint64_t)cam->width * cam->height;
    const uint64_t end_sample = (uint64_t)first_sample + p->spp;
    if (npix == 0 || npix * end_sample > 0xFFFFFFFFull)
        return fail(RB2_EINVAL, "image x (first sample + spp) must fit 32-bit sample keys");
    // Samples per pixel in flight: up to kRenderWavePaths paths per wave by default.
    const uint64_t P = pt_paths_in_flight(npix, p->spp, p->spp_per_wave, it->wave_paths ? it->wave_paths : kRenderWavePaths);
    const uint32_t spw = (uint32_t)(P / npix);
    PathState& ps = it->ps;
    int rc;
    if ((rc = ensure_path_state(ps, P))) return rc;
    const bool filtered = it->filter.kind != RB2_FILTER_NONE;
    rb2dev::FilmArgs fa{};
    if (filtered) {
        if ((rc = grow(it->d_film_xy, it->cap_film_xy, P))) return rc;
        if ((rc = film_args(it->filter, cam->width, cam->height, fa))) return rc;
    }
    if (!it->d_wave) RB2_CUDA(rb2::dev_malloc(&it->d_wave, sizeof(WaveCounters)), "wave counters");
    if (reset) RB2_CUDA(cudaMemsetAsync(accum, 0, npix * 16, s), "accumulator reset");
    RB2_CUDA(cudaMemsetAsync(it->d_wave, 0, sizeof(WaveCounters), s), "counter reset");

    rb2dev::CamArgs ca;
    std::memcpy(ca.r2c, cam->raster_to_camera, sizeof(ca.r2c));
    std::memcpy(ca.c2w, cam->camera_to_world, sizeof(ca.c2w));
    ca.width = cam->width; ca.height = cam->height; ca.spp = 1; ca.jitter = 1; ca.seed = p->seed;
    const rb2_scene_dev* sd = it->scene;
    rb2dev::SceneView sv{sd->d_verts, sd->d_tris, sd->d_albedo, sd->d_emission, sd->d_lights, sd->n_lights, sd->d_mats};
    const DeviceBvhView bv = device_bvh(it->tracer, true);
    const DeviceBvhView bv_cam = device_bvh(it->tracer, cw8_origin_ok(it->tracer, cam->eye));
    WaveCounters* wc = it->d_wave;
    const unsigned g = grid_for(P, it->sms);
    // (The step stops at the end instead of stepping past it, so a count of
    // samples near 2^32 cannot wrap the counter.)
    for (uint32_t s0 = first_sample; s0 < (uint32_t)end_sample;
         s0 = (uint32_t)end_sample - s0 > spw ? s0 + spw : (uint32_t)end_sample) {
        const uint32_t cur_spw = std::min(spw, (uint32_t)end_sample - s0);
        const uint32_t paths = (uint32_t)(npix * cur_spw);
        rb2dev::k_pt_camera<<<g, 256, 0, s>>>(ca, p->seed, (uint32_t)npix, paths, s0, ps.ray, ps.T, ps.L, ps.q[0], wc,
                                              filtered ? it->d_film_xy : nullptr);
        RB2_CUDA(cudaGetLastError(), "PT camera");
        uint32_t cur = 0;
        for (uint32_t b = 0; b <= p->max_depth; b++) {
            rb2dev::k_pt_bounce_reset<<<1, 1, 0, s>>>(wc, cur ^ 1u);
            const DeviceBvhView& bx = b == 0 ? bv_cam : bv;  // camera rays: see cw8_origin_ok
            rb2dev::QueueSource ext{static_cast<const float4*>(bx.nodes), static_cast<const float4*>(bx.woop), bx.triidx,
                                    ps.q[cur], &wc->n_ext[cur], ps.ray, &wc->head_ext, rb2dev::kClosest,
                                    ps.hit, nullptr, nullptr};
            if ((rc = launch_persistent(ext, paths, it, bx, s))) return rc;
            rb2dev::k_pt_shade<<<g, 256, 0, s>>>(sv, p->seed, (uint32_t)npix, s0, b, p->max_depth, p->rr_start, p->rr_prob,
                                                p->compat, ps.q[cur], ps.q[cur ^ 1u], ps.ray, ps.hit, ps.T, ps.L,
                                                ps.sray, ps.sc, ps.qs, wc, cur);
            RB2_CUDA(cudaGetLastError(), "PT shade");
            rb2dev::k_pt_stats_shadow<<<1, 1, 0, s>>>(wc);
            rb2dev::QueueSource shadow{static_cast<const float4*>(bv.nodes), static_cast<const float4*>(bv.woop),
                                       bv.triidx, ps.qs, &wc->n_shadow, ps.sray, &wc->head_shadow,
                                       rb2dev::kOcclusion, nullptr, ps.L, ps.sc};
            if ((rc = launch_persistent(shadow, paths, it, bv, s))) return rc;
            cur ^= 1u;
        }
        if (filtered)
            rb2dev::k_film_gather<<<grid_for(npix, it->sms), 256, 0, s>>>(
                fa, rb2dev::ArrayPos{it->d_film_xy, (uint32_t)npix}, ps.L, cur_spw, accum, nullptr);
        else
            rb2dev::k_pt_accumulate<<<grid_for(npix, it->sms), 256, 0, s>>>(ps.L, (uint32_t)npix, cur_spw, accum);
        RB2_CUDA(cudaGetLastError(), "PT accumulate");
    }
    if (!d_rgb) return RB2_OK;
    if (filtered)
        rb2dev::k_film_resolve<<<grid_for(npix, it->sms), 256, 0, s>>>(accum, (uint32_t)npix, d_rgb);
    else
        rb2dev::k_pt_finalize<<<grid_for(npix, it->sms), 256, 0, s>>>(accum, (uint32_t)npix,
                                                                      1.0f / (float)end_sample, d_rgb);
    RB2_CUDA(cudaGetLastError(), "PT finalize");
    return RB2_OK;
}

}  // namespace

int rb2_render_pt(rb2_integrator* it, const rb2_camera* cam, const rb2_pt_params* p, float* d_rgb, void* stream)
{
    if (!it || !cam || !p || !d_rgb) return fail(RB2_EINVAL, "null argument");
    const uint64_t npix = (uint64_t)cam->width * cam->height;
    if (npix && npix <= 0xFFFFFFFFull) {
        if (int rc = grow(it->d_accum, it->cap_accum, npix)) return rc;
    }
    return render_pt(it, cam, p, 0, it->d_accum, true, d_rgb, stream);
}

int rb2_render_pt_progressive(rb2_integrator* it, const rb2_camera* cam, const rb2_pt_params* p, uint32_t first_sample,
                              float* d_sum, float* d_rgb, void* stream)
{
    if (!it || !cam || !p || !d_sum) return fail(RB2_EINVAL, "null argument");
    if ((uintptr_t)d_sum & 15u) return fail(RB2_EINVAL, "d_sum must be 16-byte aligned");
    return render_pt(it, cam, p, first_sample, reinterpret_cast<float4*>(d_sum), false, d_rgb, stream);
}

int rb2_render_raycast(rb2_integrator* it, const rb2_camera* cam, const rb2_raycast_params* p, float* d_rgb,
                       void* stream)
{
    rb2::Range nvtx_range("rb2_render_raycast");
    if (!it || !cam || !p || !d_rgb) return fail(RB2_EINVAL, "null argument");
    it->ev_used = 0;
    if (p->spp == 0) return fail(RB2_EINVAL, "spp must be > 0");
    if (p->shade > RB2_RAYCAST_SHADE_UNIFORM) return fail(RB2_EINVAL, "shade must be an RB2_RAYCAST_SHADE_* value");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t npix = (uint64_t)cam->width * cam->height;
    if (npix == 0 || npix * p->spp > 0xFFFFFFFFull) return fail(RB2_EINVAL, "image x spp must fit 32-bit sample keys");
    const uint64_t P = pt_paths_in_flight(npix, p->spp, 0, it->wave_paths ? it->wave_paths : kRenderWavePaths);
    const uint32_t spw = (uint32_t)(P / npix);
    PathState& ps = it->ps;
    int rc;
    if ((rc = ensure_path_state(ps, P))) return rc;
    if ((rc = grow(it->d_accum, it->cap_accum, npix))) return rc;
    const bool filtered = it->filter.kind != RB2_FILTER_NONE;
    rb2dev::FilmArgs fa{};
    if (filtered) {
        if ((rc = grow(it->d_film_xy, it->cap_film_xy, P))) return rc;
        if ((rc = film_args(it->filter, cam->width, cam->height, fa))) return rc;
    }
    if (!it->d_wave) RB2_CUDA(rb2::dev_malloc(&it->d_wave, sizeof(WaveCounters)), "wave counters");
    RB2_CUDA(cudaMemsetAsync(it->d_accum, 0, npix * 16, s), "accumulator reset");
    RB2_CUDA(cudaMemsetAsync(it->d_wave, 0, sizeof(WaveCounters), s), "counter reset");
    rb2dev::CamArgs ca;
    std::memcpy(ca.r2c, cam->raster_to_camera, sizeof(ca.r2c));
    std::memcpy(ca.c2w, cam->camera_to_world, sizeof(ca.c2w));
    ca.width = cam->width; ca.height = cam->height; ca.spp = 1; ca.jitter = 1; ca.seed = p->seed;
    const rb2_scene_dev* sd = it->scene;
    rb2dev::SceneView sv{sd->d_verts, sd->d_tris, sd->d_albedo, sd->d_emission, sd->d_lights, sd->n_lights, sd->d_mats};
    const DeviceBvhView bv = device_bvh(it->tracer, true);
    const DeviceBvhView bv_cam = device_bvh(it->tracer, cw8_origin_ok(it->tracer, cam->eye));
    WaveCounters* wc = it->d_wave;
    const unsigned g = grid_for(P, it->sms);
    for (uint32_t s0 = 0; s0 < p->spp; s0 = p->spp - s0 > spw ? s0 + spw : p->spp) {
        const uint32_t cur_spw = std::min(spw, p->spp - s0);
        const uint32_t paths = (uint32_t)(npix * cur_spw);
        // Camera samples (kernel_generate_perspective_camera_samples), then the
        // closest-hit trace (CudaTracer::trace with any_hit = false).
        rb2dev::k_pt_camera<<<g, 256, 0, s>>>(ca, p->seed, (uint32_t)npix, paths, s0, ps.ray, nullptr, nullptr, ps.q[0],
                                              wc, filtered ? it->d_film_xy : nullptr);
        RB2_CUDA(cudaGetLastError(), "ray-cast camera");
        rb2dev::k_pt_bounce_reset<<<1, 1, 0, s>>>(wc, 1u);
        rb2dev::QueueSource prim{static_cast<const float4*>(bv_cam.nodes), static_cast<const float4*>(bv_cam.woop),
                                 bv_cam.triidx, ps.q[0], &wc->n_ext[0], ps.ray, &wc->head_ext, rb2dev::kClosest,
                                 ps.hit, nullptr, nullptr};
        if ((rc = launch_persistent(prim, paths, it, bv_cam, s))) return rc;
        if (filtered) {
            rb2dev::k_rc_shade<<<g, 256, 0, s>>>(sv, paths, p->shade, ps.hit, ps.L, wc);
            rb2dev::k_film_gather<<<grid_for(npix, it->sms), 256, 0, s>>>(
                fa, rb2dev::ArrayPos{it->d_film_xy, (uint32_t)npix}, ps.L, cur_spw, it->d_accum, nullptr);
        } else {
            rb2dev::k_rc_shade_accumulate<<<grid_for(npix, it->sms), 256, 0, s>>>(sv, (uint32_t)npix, cur_spw, p->shade,
                                                                                 ps.hit, it->d_accum, wc);
        }
        RB2_CUDA(cudaGetLastError(), "ray-cast shade");
    }
    if (filtered)
        rb2dev::k_film_resolve<<<grid_for(npix, it->sms), 256, 0, s>>>(it->d_accum, (uint32_t)npix, d_rgb);
    else
        rb2dev::k_pt_finalize<<<grid_for(npix, it->sms), 256, 0, s>>>(it->d_accum, (uint32_t)npix, 1.0f / (float)p->spp,
                                                                      d_rgb);
    RB2_CUDA(cudaGetLastError(), "ray-cast finalize");
    return RB2_OK;
}

int rb2_render_bdpt(rb2_integrator* it, const rb2_camera* cam, const rb2_bdpt_params* p, float* d_rgb, void* stream)
{
    rb2::Range nvtx_range("rb2_render_bdpt");
    if (!it || !cam || !p || !d_rgb) return fail(RB2_EINVAL, "null argument");
    rb2_bdpt_lvc_params q{};
    q.spp = p->spp;
    q.num_light_paths = p->num_light_paths;
    q.light_path_rrstart = p->rr_start;
    q.cam_path_rrstart = p->rr_start;
    q.cam_path_rrprob = p->rr_prob;
    q.num_cam_path_connections = p->connections;
    q.estimator = RB2_BDPT_ESTIMATOR_UNBIASED;
    q.max_path_length = p->max_path_length;
    q.seed = p->seed;
    return rb2_render_bdpt_lvc(it, cam, &q, d_rgb, stream);
}

int rb2_render_bdpt_lvc(rb2_integrator* it, const rb2_camera* cam, const rb2_bdpt_lvc_params* p, float* d_rgb,
                        void* stream)
{
    rb2::Range nvtx_range("rb2_render_bdpt_lvc");
    if (!it || !cam || !p || !d_rgb) return fail(RB2_EINVAL, "null argument");
    it->ev_used = 0;
    if (p->spp == 0) return fail(RB2_EINVAL, "spp must be > 0");
    if (p->estimator > RB2_BDPT_ESTIMATOR_REFERENCE) return fail(RB2_EINVAL, "unknown BDPT estimator");
    if (p->mode > RB2_BDPT_MODE_SORT) return fail(RB2_EINVAL, "unknown BDPT mode (sk, mk, sort)");
    const bool ref = p->estimator == RB2_BDPT_ESTIMATOR_REFERENCE;
    if (!ref && (p->max_path_length < 1 || p->max_path_length > 16))
        return fail(RB2_EINVAL, "max_path_length must be in [1, 16]");
    if (ref && (p->num_light_path_max_depth < 1 || p->num_light_path_max_depth > 16))
        return fail(RB2_EINVAL, "num_light_path_max_depth must be in [1, 16] (it bounds the light-vertex cache)");
    if (ref && p->num_cam_path_max_depth > 63) return fail(RB2_EINVAL, "num_cam_path_max_depth must be <= 63");
    if (ref && !(p->cam_path_rrprob < 1.0f))
        return fail(RB2_EINVAL, "the reference estimator divides by 1 - q: cam_path_rrprob must be < 1");
    if (p->num_cam_path_connections < 1 || p->num_cam_path_connections > rb2dev::kMaxConnections)
        return fail(RB2_EINVAL, "num_cam_path_connections must be in [1, 8]");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t npix = (uint64_t)cam->width * cam->height;
    if (npix == 0 || npix * p->spp > 0xFFFFFFFFull) return fail(RB2_EINVAL, "image x spp must fit 32-bit sample keys");
    // K: camera vertices of a path (unbiased: the whole-path cap in segments,
    // which also bounds the camera subpath; reference: bounces 0..max depth).
    const uint32_t K = ref ? p->num_cam_path_max_depth + 1 : p->max_path_length;
    const uint32_t C = p->num_cam_path_connections;
    // Connection-ray slots per camera vertex (the reference estimator adds the
    // BSDF half of its NEE as one more occlusion segment).
    const uint32_t Cs = ref ? C + 1 : C;
    // Cached light vertices per subpath: y1..y_{K-2} suffice for paths of at most
    // K segments; the reference estimator keeps up to num_light_path_max_depth.
    const uint32_t Dl = ref ? p->num_light_path_max_depth : (K >= 2 ? K - 2 : 0);
    const uint64_t NL = p->num_light_paths ? p->num_light_paths : npix;
    const uint32_t rr_light = p->light_path_rrstart, rr_cam = p->cam_path_rrstart;
    const float rr_prob = p->cam_path_rrprob;
    // Iterations per wave: as many as fit the wave budget in camera and light
    // paths, spread evenly over the waves, with every wave index 32-bit.
    const uint64_t per_iter = NL * std::max<uint32_t>(Dl, 1);   // cache slots of one iteration
    if (per_iter > 0xFFFFFFFFull) return fail(RB2_EINVAL, "num_light_paths x cached depth must fit 32-bit slot indices");
    const uint64_t budget = it->wave_paths ? it->wave_paths : kBdptWavePaths;
    uint64_t wmax = std::max<uint64_t>(1, budget / std::max(npix, NL));
    wmax = std::min<uint64_t>({wmax, (uint64_t)p->spp, (uint64_t)kMaxBdptWave, 0xFFFFFFFFull / (npix * Cs),
                               0xFFFFFFFFull / per_iter});
    wmax = std::max<uint64_t>(wmax, 1);
    const uint32_t n_waves = (uint32_t)((p->spp + wmax - 1) / wmax);
    const uint32_t Wv = (p->spp + n_waves - 1) / n_waves;
    const uint64_t n_slots = per_iter * Wv;
    // The reference estimator's preparation pass traces num_prep_paths light
    // subpaths through the same buffers (integrator_bdpt_lvc_sk.cu:447-470).
    const uint64_t n_prep = ref ? p->num_prep_paths : 0;
    if (n_prep * std::max<uint32_t>(Dl, 1) > 0xFFFFFFFFull)
        return fail(RB2_EINVAL, "num_prep_paths x cached depth must fit 32-bit slot indices");
    int rc;
    if ((rc = ensure_path_state(it->ps, npix * Wv))) return rc;
    if ((rc = ensure_bdpt_state(it->bd, std::max<uint64_t>(NL * Wv, n_prep),
                                std::max<uint64_t>(n_slots, n_prep * std::max<uint32_t>(Dl, 1)), npix * Wv * Cs)))
        return rc;
    if ((rc = grow(it->d_accum, it->cap_accum, npix))) return rc;
    const bool filtered = it->filter.kind != RB2_FILTER_NONE;
    rb2dev::FilmArgs fa{};
    if (filtered) {
        if ((rc = grow(it->d_film_xy, it->cap_film_xy, npix * Wv))) return rc;
        if ((rc = film_args(it->filter, cam->width, cam->height, fa))) return rc;
    }
    if (!it->d_wave) RB2_CUDA(rb2::dev_malloc(&it->d_wave, sizeof(WaveCounters)), "wave counters");
    RB2_CUDA(cudaMemsetAsync(it->d_accum, 0, npix * 16, s), "accumulator reset");
    RB2_CUDA(cudaMemsetAsync(it->d_wave, 0, sizeof(WaveCounters), s), "counter reset");

    rb2dev::CamArgs ca;
    std::memcpy(ca.r2c, cam->raster_to_camera, sizeof(ca.r2c));
    std::memcpy(ca.c2w, cam->camera_to_world, sizeof(ca.c2w));
    ca.width = cam->width; ca.height = cam->height; ca.spp = 1; ca.jitter = 1; ca.seed = p->seed;
    const rb2_scene_dev* sd = it->scene;
    rb2dev::SceneView sv{sd->d_verts, sd->d_tris, sd->d_albedo, sd->d_emission, sd->d_lights, sd->n_lights, sd->d_mats};
    const DeviceBvhView bv = device_bvh(it->tracer, true);
    const DeviceBvhView bv_cam = device_bvh(it->tracer, cw8_origin_ok(it->tracer, cam->eye));
    const float4* bn = static_cast<const float4*>(bv.nodes);
    const float4* bw = static_cast<const float4*>(bv.woop);
    WaveCounters* wc = it->d_wave;
    PathState& ps = it->ps;
    BdptState& bd = it->bd;
    // Light-vertex directions are cached only when a layered material needs them.
    float4* s_wi = it->scene->layered ? bd.s_wi : nullptr;
    // Light subpaths of a wave (or of the preparation pass) into the sparse cache.
    auto light_pass = [&](uint64_t key0, uint64_t n_light) -> int {
        const unsigned gl = grid_for(n_light, it->sms);
        RB2_CUDA(cudaMemsetAsync(bd.s_valid, 0, n_light * std::max<uint32_t>(Dl, 1), s), "cache reset");
        if (ref)
            rb2dev::k_bd_light_init_ref<<<gl, 256, 0, s>>>(sv, p->seed, key0, (uint32_t)n_light, bd.lray, bd.lbeta,
                                                           bd.lq[0], wc);
        else
            rb2dev::k_bd_light_init<<<gl, 256, 0, s>>>(sv, p->seed, key0, (uint32_t)n_light, bd.lray, bd.lbeta,
                                                       bd.lq[0], wc);
        RB2_CUDA(cudaGetLastError(), "BDPT light init");
        uint32_t lc = 0;
        for (uint32_t d = 1; d <= Dl; d++) {
            rb2dev::k_pt_bounce_reset<<<1, 1, 0, s>>>(wc, lc ^ 1u);
            rb2dev::QueueSource lsrc{bn, bw, bv.triidx, bd.lq[lc], &wc->n_ext[lc], bd.lray, &wc->head_ext,
                                     rb2dev::kClosest, bd.lhit, nullptr, nullptr};
            int r = launch_persistent(lsrc, n_light, it, bv, s);
            if (r) return r;
            if (ref)
                rb2dev::k_bd_light_shade_ref<<<gl, 256, 0, s>>>(sv, p->seed, key0, d, Dl, bd.lq[lc], bd.lq[lc ^ 1u],
                                                                bd.lray, bd.lhit, bd.lbeta, bd.s_pos, bd.s_nrm,
                                                                bd.s_beta, s_wi, bd.s_valid, wc, lc);
            else
                rb2dev::k_bd_light_shade<<<gl, 256, 0, s>>>(sv, p->seed, key0, d, Dl, rr_light, rr_prob, bd.lq[lc],
                                                            bd.lq[lc ^ 1u], bd.lray, bd.lhit, bd.lbeta, bd.s_pos,
                                                            bd.s_nrm, bd.s_beta, s_wi, bd.s_valid, wc, lc);
            RB2_CUDA(cudaGetLastError(), "BDPT light shade");
            lc ^= 1u;
        }
        return RB2_OK;
    };
    // Cache capacity of one iteration (reference estimator): 1.1 x the mean
    // number of vertices a preparation subpath stored x num_light_paths, in
    // single precision as the reference computes it (integrator_bdpt_lvc_sk.cu:466-470).
    uint32_t lvc_cap = 0xFFFFFFFFu;
    if (n_prep > 0) {
        if ((rc = light_pass((uint64_t)p->spp * NL, n_prep))) return rc;
        const uint64_t prep_slots = n_prep * Dl;
        const uint64_t n_chunks = (prep_slots + rb2dev::kScanChunk - 1) / rb2dev::kScanChunk;
        rb2dev::k_lvc_count<<<(unsigned)n_chunks, rb2dev::kScanThreads, 0, s>>>(bd.s_valid, prep_slots, bd.block_sums);
        rb2dev::k_lvc_scan_top<<<1, 1024, 0, s>>>(bd.block_sums, (uint32_t)n_chunks, wc);
        RB2_CUDA(cudaGetLastError(), "preparation count");
        uint32_t total = 0;
        RB2_CUDA(cudaMemcpyAsync(&total, &wc->lvc_count, sizeof(total), cudaMemcpyDeviceToHost, s), "preparation read");
        RB2_CUDA(cudaStreamSynchronize(s), "preparation sync");
        const float avg = (float)total / (float)n_prep;
        const float cap = std::ceil(1.1f * avg * (float)NL);
        lvc_cap = cap >= 4294967295.0f ? 0xFFFFFFFFu : (uint32_t)cap;
    }
    for (uint32_t it0 = 0; it0 < p->spp; it0 = p->spp - it0 > Wv ? it0 + Wv : p->spp) {
        // Wave of w iterations: light path l is path l % NL of iteration it0 + l / NL,
        // camera path c is pixel c % npix of iteration it0 + c / npix.  The random
        // keys are those of the iterations run one at a time.
        const uint32_t w = std::min(Wv, p->spp - it0);
        const uint64_t n_light = NL * w, n_cam = npix * w, wave_slots = per_iter * w;
        const unsigned gc = grid_for(n_cam, it->sms), gp = grid_for(npix, it->sms);
        const uint64_t n_chunks = (wave_slots + rb2dev::kScanChunk - 1) / rb2dev::kScanChunk;
        // ---- light pass: subpaths into the sparse cache, then compaction.
        if ((rc = light_pass((uint64_t)it0 * NL, n_light))) return rc;
        uint32_t cur = 0;
        rb2dev::k_lvc_count<<<(unsigned)n_chunks, rb2dev::kScanThreads, 0, s>>>(bd.s_valid, wave_slots, bd.block_sums);
        rb2dev::k_lvc_scan_top<<<1, 1024, 0, s>>>(bd.block_sums, (uint32_t)n_chunks, wc);
        rb2dev::k_lvc_scatter<<<(unsigned)n_chunks, rb2dev::kScanThreads, 0, s>>>(
            bd.s_valid, wave_slots, bd.block_sums, bd.d_slot);
        rb2dev::k_lvc_wave_offsets<<<w + 1, rb2dev::kScanThreads, 0, s>>>(bd.s_valid, wave_slots, bd.block_sums,
                                                                          per_iter, wc, bd.lvc_off);
        RB2_CUDA(cudaGetLastError(), "cache compaction");
        // ---- camera pass.
        rb2dev::k_pt_camera<<<gc, 256, 0, s>>>(ca, p->seed, (uint32_t)npix, (uint32_t)n_cam, it0, ps.ray, ps.T, ps.L,
                                               ps.q[0], wc, filtered ? it->d_film_xy : nullptr);
        RB2_CUDA(cudaGetLastError(), "BDPT camera");
        cur = 0;
        for (uint32_t i = 1; i <= K; i++) {
            rb2dev::k_pt_bounce_reset<<<1, 1, 0, s>>>(wc, cur ^ 1u);
            const DeviceBvhView& bx = i == 1 ? bv_cam : bv;  // camera rays: see cw8_origin_ok
            rb2dev::QueueSource ext{static_cast<const float4*>(bx.nodes), static_cast<const float4*>(bx.woop), bx.triidx,
                                    ps.q[cur], &wc->n_ext[cur], ps.ray, &wc->head_ext, rb2dev::kClosest, ps.hit,
                                    nullptr, nullptr};
            if ((rc = launch_persistent(ext, n_cam, it, bx, s))) return rc;
            if (ref)
                rb2dev::k_bd_cam_shade_ref<<<gc, 256, 0, s>>>(sv, p->seed, (uint32_t)npix, it0, i, K, C, Cs, rr_cam,
                                                              rr_prob, lvc_cap, ps.q[cur], ps.q[cur ^ 1u], ps.ray, ps.hit, ps.T,
                                                              ps.L, ps.sray, ps.sc, ps.qs, bd.cray, bd.cc, bd.cq,
                                                              bd.s_pos, bd.s_nrm, bd.s_beta, s_wi, bd.d_slot,
                                                              bd.lvc_off, wc, cur);
            else
                rb2dev::k_bd_cam_shade<<<gc, 256, 0, s>>>(sv, p->seed, (uint32_t)npix, it0, i, K, C, rr_cam, rr_prob,
                                                          (float)NL, ps.q[cur], ps.q[cur ^ 1u], ps.ray, ps.hit, ps.T,
                                                          ps.L, ps.sray, ps.sc, ps.qs, bd.cray, bd.cc, bd.cq, bd.s_pos,
                                                          bd.s_nrm, bd.s_beta, s_wi, bd.d_slot, bd.lvc_off, wc, cur);
            RB2_CUDA(cudaGetLastError(), "BDPT camera shade");
            rb2dev::k_bd_stats<<<1, 1, 0, s>>>(wc);
            rb2dev::QueueSource nee{bn, bw, bv.triidx, ps.qs, &wc->n_shadow, ps.sray, &wc->head_shadow,
                                    rb2dev::kOcclusion, nullptr, ps.L, ps.sc};
            if ((rc = launch_persistent(nee, n_cam, it, bv, s))) return rc;
            rb2dev::QueueSource con{bn, bw, bv.triidx, bd.cq, &wc->n_conn, bd.cray, &wc->head_conn,
                                    rb2dev::kOcclusion, nullptr, nullptr, bd.cc};
            if ((rc = launch_persistent(con, n_cam * Cs, it, bv, s))) return rc;
            rb2dev::k_bd_conn_reduce<<<gc, 256, 0, s>>>(ps.q[cur], wc, cur, Cs, bd.cc, ps.L);
            RB2_CUDA(cudaGetLastError(), "BDPT connection reduce");
            cur ^= 1u;
        }
        // Unfiltered, the iterations are added to the accumulator in order, so the
        // image is bit-identical to running them one at a time; the filtered
        // gather sums a neighbourhood sample by sample, so its rounding depends
        // on the wave size (and is deterministic for a given one).
        if (filtered)
            rb2dev::k_film_gather<<<gp, 256, 0, s>>>(fa, rb2dev::ArrayPos{it->d_film_xy, (uint32_t)npix}, ps.L, w,
                                                     it->d_accum, nullptr);
        else
            rb2dev::k_pt_accumulate<<<gp, 256, 0, s>>>(ps.L, (uint32_t)npix, w, it->d_accum);
        RB2_CUDA(cudaGetLastError(), "BDPT accumulate");
    }
    const unsigned gp = grid_for(npix, it->sms);
    if (filtered)
        rb2dev::k_film_resolve<<<gp, 256, 0, s>>>(it->d_accum, (uint32_t)npix, d_rgb);
    else
        rb2dev::k_pt_finalize<<<gp, 256, 0, s>>>(it->d_accum, (uint32_t)npix, 1.0f / (float)p->spp, d_rgb);
    RB2_CUDA(cudaGetLastError(), "BDPT finalize");
    return RB2_OK;
}

int rb2_integrator_stats(rb2_integrator* it, rb2_render_stats* out, void* stream)
{
    if (!it || !out) return fail(RB2_EINVAL, "null argument");
    std::memset(out, 0, sizeof(*out));
    if (it->timing) {
        double ms = 0.0;
        for (uint32_t k = 0; k + 1 < it->ev_used; k += 2) {
            float e = 0.0f;
            RB2_CUDA(cudaEventSynchronize(it->ev[k + 1]), "timing sync");
            RB2_CUDA(cudaEventElapsedTime(&e, it->ev[k], it->ev[k + 1]), "timing read");
            ms += e;
        }
        out->trace_ms = ms;
    }
    if (!it->d_wave) return RB2_OK;
    WaveCounters w;
    cudaStream_t s = (cudaStream_t)stream;
    RB2_CUDA(cudaMemcpyAsync(&w, it->d_wave, sizeof(w), cudaMemcpyDeviceToHost, s), "stats read");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    out->primary_rays = w.stats[0];
    out->extension_rays = w.stats[1];
    out->shadow_rays = w.stats[2];
    out->connection_rays = w.stats[3];
    out->light_rays = w.stats[4];
    out->lvc_vertices = w.stats[5];
    return RB2_OK;
}

int rb2_integrator_set_wave(rb2_integrator* it, uint64_t paths)
{
    if (!it) return fail(RB2_EINVAL, "null argument");
    it->wave_paths = paths;
    return RB2_OK;
}

int rb2_integrator_set_timing(rb2_integrator* it, int on)
{
    if (!it) return fail(RB2_EINVAL, "null argument");
    it->timing = on != 0;
    it->ev_used = 0;
    return RB2_OK;
}

}  // extern "C"
