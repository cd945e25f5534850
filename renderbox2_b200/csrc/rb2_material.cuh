// Layered materials on the device: the reference's BSDFs
// (core/reflection.cu:42-299, core/reflection.h:82-212) and the material
// dispatch (core/material.cu:56-326), in the local shading frame whose z is
// the (unflipped) geometric normal, as Frame::set_from_z(Ns) builds it.
// Differences from the reference, applied identically by the oracle: the
// pdf of a multi-layer material is divided by the number of layers when a
// direction is sampled (pbrt-v2 semantics; the reference kept the sum), and
// a glass layer contributes no microfacet term (missing `break`, Q11).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb2_shading.cuh"

namespace rb2dev {

constexpr uint32_t kMaxLayers = 4;
enum BsdfKind : uint32_t { kLambertian = 0, kOrenNayar = 1, kMirror = 2, kGlass = 3, kMicrofacet = 4 };
enum FresnelKind : uint32_t { kFresnelDielectric = 0, kFresnelConductor = 1, kFresnelNoop = 2 };

// One layer, 64 bytes: q0 = (color, exponent), q1 = (eta, etai),
// q2 = (k, etat), q3 = (A, B, kind bits, fresnel bits).
struct LayerDev {
    float4 q0, q1, q2, q3;
};
// flags: bit 0 = a single Lambertian layer (the integrators' fast path),
// bit 1 = has a non-specular layer (next-event estimation applies).
struct MaterialDev {
    uint32_t n_layers, flags, pad0, pad1;
    LayerDev layer[kMaxLayers];
};
constexpr uint32_t kMatPlainLambertian = 1u, kMatHasNonDelta = 2u;

__device__ __forceinline__ uint32_t layer_kind(const LayerDev& l) { return __float_as_uint(l.q3.z); }
__device__ __forceinline__ bool kind_is_delta(uint32_t k) { return k == kMirror || k == kGlass; }

// BxDF type bits as the scene reader assigns them (io/customfilereader.cpp:113-204).
enum : uint32_t { kRefl = 1u, kTrans = 2u, kDiffuse = 4u, kGlossy = 8u, kSpecular = 16u };
__device__ __forceinline__ uint32_t bxdf_bits(uint32_t k)
{
    switch (k) {
    case kMirror: return kRefl | kSpecular;
    case kGlass: return kRefl | kSpecular | kTrans;
    case kMicrofacet: return kRefl | kGlossy;
    default: return kRefl | kDiffuse;
    }
}

// ---- shading-frame helpers (core/reflection.h:67-140) ---------------------------------
__device__ __forceinline__ float sin2_theta(float3 w) { return fmaxf(0.0f, 1.0f - w.z * w.z); }
__device__ __forceinline__ float sin_theta_of(float3 w) { return sqrtf(sin2_theta(w)); }
__device__ __forceinline__ float cos_phi_of(float3 w)
{
    const float s = sin_theta_of(w);
    return s == 0.0f ? 1.0f : fminf(fmaxf(w.x / s, -1.0f), 1.0f);
}
__device__ __forceinline__ float sin_phi_of(float3 w)
{
    const float s = sin_theta_of(w);
    return s == 0.0f ? 0.0f : fminf(fmaxf(w.y / s, -1.0f), 1.0f);
}
__device__ __forceinline__ bool same_hemi(float3 a, float3 b) { return a.z * b.z > 0.0f; }
__device__ __forceinline__ float3 unit(float3 v) { return mul(v, 1.0f / sqrtf(dot3(v, v))); }
__device__ __forceinline__ float3 to_local(const Frame& f, float3 w) { return f3(dot3(w, f.x), dot3(w, f.y), dot3(w, f.z)); }

// Fresnel terms (core/reflection.h:146-212).
__device__ __forceinline__ float3 fresnel_dielectric_eval(float cosi, float etai_, float etat_)
{
    const bool entering = cosi > 0.0f;
    const float ei = entering ? etai_ : etat_, et = entering ? etat_ : etai_;
    const float sint = ei / et * sqrtf(fmaxf(0.0f, 1.0f - cosi * cosi));
    if (sint >= 1.0f) return f3(1.0f, 1.0f, 1.0f);
    const float cost = sqrtf(fmaxf(0.0f, 1.0f - sint * sint));
    const float ci = fabsf(cosi);
    const float rpar = (et * ci - ei * cost) / (et * ci + ei * cost);
    const float rperp = (ei * ci - et * cost) / (ei * ci + et * cost);
    const float r = (rpar * rpar + rperp * rperp) / 2.0f;
    return f3(r, r, r);
}
__device__ __forceinline__ float fresnel_conductor1(float cosi, float eta, float k)
{
    const float tmp = (eta * eta + k * k) * cosi * cosi;
    const float rpar2 = (tmp - 2.0f * eta * cosi + 1.0f) / (tmp + 2.0f * eta * cosi + 1.0f);
    const float tf = eta * eta + k * k;
    const float rperp2 = (tf - 2.0f * eta * cosi + cosi * cosi) / (tf + 2.0f * eta * cosi + cosi * cosi);
    return (rpar2 + rperp2) / 2.0f;
}
__device__ __forceinline__ float3 fresnel_eval(const LayerDev& l, float cosi)
{
    const uint32_t t = __float_as_uint(l.q3.w);
    if (t == kFresnelConductor)
        return f3(fresnel_conductor1(cosi, l.q1.x, l.q2.x), fresnel_conductor1(cosi, l.q1.y, l.q2.y),
                  fresnel_conductor1(cosi, l.q1.z, l.q2.z));
    if (t == kFresnelDielectric) return fresnel_dielectric_eval(fminf(fmaxf(cosi, -1.0f), 1.0f), l.q1.w, l.q2.w);
    return f3(1.0f, 1.0f, 1.0f);
}

// ---- per-layer evaluation (local frame) --------------------------------------------
__device__ __forceinline__ float blinn_D(float3 wh, float e)
{
    return (e + 2.0f) * (0.5f * kInvPi) * powf(fabsf(wh.z), e);
}
__device__ __forceinline__ float blinn_pdf(float3 wo, float3 wi, float e)
{
    const float3 wh = unit(add(wo, wi));
    const float c = fabsf(wh.z);
    const float d = dot3(wo, wh);
    if (d <= 0.0f) return 0.0f;
    return ((e + 1.0f) * powf(c, e)) / (2.0f * 3.14159265358979323846f * 4.0f * d);
}
__device__ __forceinline__ float3 eval_microfacet(const LayerDev& l, float3 wi, float3 wo)
{
    const float co = fabsf(wo.z), ci = fabsf(wi.z);
    if (ci == 0.0f || co == 0.0f) return f3(0.0f, 0.0f, 0.0f);
    float3 wh = add(wi, wo);
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return f3(0.0f, 0.0f, 0.0f);
    wh = unit(wh);
    const float3 F = fresnel_eval(l, dot3(wi, wh));
    const float nh = fabsf(wh.z), woh = fabsf(dot3(wo, wh));
    const float G = fminf(1.0f, fminf(2.0f * nh / woh, 2.0f * nh * ci / woh));  // microfacet_G as written
    const float s = blinn_D(wh, l.q0.w) * G / (4.0f * ci * co);
    return f3(l.q0.x * s * F.x, l.q0.y * s * F.y, l.q0.z * s * F.z);
}
__device__ __forceinline__ float3 eval_orennayar(const LayerDev& l, float3 wi, float3 wo)
{
    const float si = sin_theta_of(wi), so = sin_theta_of(wo);
    float maxcos = 0.0f;
    if (si > 1e-4f && so > 1e-4f)
        maxcos = fmaxf(0.0f, cos_phi_of(wi) * cos_phi_of(wo) + sin_phi_of(wi) * sin_phi_of(wo));
    float sinalpha, tanbeta;
    if (fabsf(wi.z) > fabsf(wo.z)) { sinalpha = so; tanbeta = si / fabsf(wi.z); }
    else { sinalpha = si; tanbeta = so / fabsf(wo.z); }
    const float s = kInvPi * (l.q3.x + l.q3.y * maxcos * sinalpha * tanbeta);
    return f3(l.q0.x * s, l.q0.y * s, l.q0.z * s);
}
// f of one layer for a non-specular evaluation (delta layers give 0).
__device__ __forceinline__ float3 layer_f(const LayerDev& l, float3 wi, float3 wo)
{
    switch (layer_kind(l)) {
    case kLambertian:
        return same_hemi(wi, wo) ? f3(l.q0.x * kInvPi, l.q0.y * kInvPi, l.q0.z * kInvPi) : f3(0.0f, 0.0f, 0.0f);
    case kOrenNayar: return eval_orennayar(l, wi, wo);
    case kMicrofacet: return eval_microfacet(l, wi, wo);
    default: return f3(0.0f, 0.0f, 0.0f);
    }
}
__device__ __forceinline__ float layer_pdf(const LayerDev& l, float3 wi, float3 wo)
{
    switch (layer_kind(l)) {
    case kLambertian:
    case kOrenNayar: return same_hemi(wi, wo) ? fabsf(wi.z) * kInvPi : 0.0f;
    case kMicrofacet: return same_hemi(wi, wo) ? blinn_pdf(wo, wi, l.q0.w) : 0.0f;
    default: return 0.0f;
    }
}

// Samples layer l: returns f, sets wi (local) and pdf; delta = mirror/glass.
__device__ __forceinline__ float3 layer_sample(const LayerDev& l, float3 wo, float u1, float u2, float3& wi, float& pdf)
{
    const uint32_t k = layer_kind(l);
    pdf = 0.0f;
    if (k == kMirror) {
        wi = f3(-wo.x, -wo.y, wo.z);
        pdf = 1.0f;
        const float s = 1.0f / fabsf(wi.z);
        return f3(l.q0.x * s, l.q0.y * s, l.q0.z * s);
    }
    if (k == kGlass) {
        const bool entering = wo.z > 0.0f;
        const float ei = entering ? l.q1.w : l.q2.w, et = entering ? l.q2.w : l.q1.w;
        const float eta = ei / et;
        const float sint2 = eta * eta * sin2_theta(wo);
        if (sint2 >= 1.0f) { wi = f3(0.0f, 0.0f, 1.0f); return f3(0.0f, 0.0f, 0.0f); }
        float cost = sqrtf(fmaxf(0.0f, 1.0f - sint2));
        if (entering) cost = -cost;
        wi = f3(eta * -wo.x, eta * -wo.y, cost);
        pdf = 1.0f;
        const float3 F = fresnel_dielectric_eval(wo.z, l.q1.w, l.q2.w);
        const float s = (et * et) / (ei * ei) / fabsf(wi.z);
        return f3(s * (1.0f - F.x) * l.q0.x, s * (1.0f - F.y) * l.q0.y, s * (1.0f - F.z) * l.q0.z);
    }
    if (k == kMicrofacet) {
        const float e = l.q0.w;
        const float ct = powf(u1, 1.0f / (e + 1.0f));
        const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float sp, cp;
        sincosf(u2 * 2.0f * 3.14159265358979323846f, &sp, &cp);
        float3 wh = f3(st * cp, st * sp, ct);
        if (!same_hemi(wo, wh)) wh = mul(wh, -1.0f);
        const float d = dot3(wo, wh);
        wi = add(mul(wo, -1.0f), mul(wh, 2.0f * d));
        pdf = d <= 0.0f ? 0.0f : ((e + 1.0f) * powf(ct, e)) / (2.0f * 3.14159265358979323846f * 4.0f * d);
        if (!same_hemi(wi, wo)) return f3(0.0f, 0.0f, 0.0f);
        return eval_microfacet(l, wi, wo);
    }
    // Lambertian / Oren-Nayar: cosine hemisphere, flipped to wo's side.
    wi = cosine_hemisphere(u1, u2);
    if (wo.z < 0.0f) wi.z = -wi.z;
    wi = unit(wi);
    pdf = same_hemi(wi, wo) ? fabsf(wi.z) * kInvPi : 0.0f;
    return layer_f(l, wi, wo);
}

// material_f (core/material.cu:254-326) with specular layers excluded: layers
// whose reflection/transmission bit disagrees with the side of wi are skipped.
__device__ __forceinline__ float3 material_f(const MaterialDev& m, float3 ng, float3 wo_w, float3 wi_w, float3 wo, float3 wi)
{
    const uint32_t side = dot3(wi_w, ng) * dot3(wo_w, ng) > 0.0f ? (kRefl | kDiffuse | kGlossy) : (kTrans | kDiffuse | kGlossy);
    float3 f = f3(0.0f, 0.0f, 0.0f);
    for (uint32_t i = 0; i < m.n_layers; i++) {
        const uint32_t bits = bxdf_bits(layer_kind(m.layer[i]));
        if ((bits & side) != bits) continue;
        f = add(f, layer_f(m.layer[i], wi, wo));
    }
    return f;
}

// material_pdf (core/material.cu:213-252) with specular layers excluded.
__device__ __forceinline__ float material_pdf(const MaterialDev& m, float3 wo, float3 wi)
{
    float pdf = 0.0f;
    uint32_t n = 0;
    for (uint32_t i = 0; i < m.n_layers; i++) {
        if (kind_is_delta(layer_kind(m.layer[i]))) continue;
        n++;
        pdf += layer_pdf(m.layer[i], wi, wo);
    }
    return n ? pdf / (float)n : 0.0f;
}

// material_sample_f (core/material.cu:56-211) over all layers.  Returns f and
// sets wi (world), pdf and whether a specular layer was sampled.
// eta_io (optional): for a sampled glass layer, the index ratio of wo's side
// to wi's side (1 for every other sample); light subpaths use it to form the
// adjoint of the transmission factor.
__device__ __forceinline__ float3 material_sample(const MaterialDev& m, const Frame& fr, float3 ng, float3 wo_w, float u1,
                                                  float u2, float uc, float3& wi_w, float& pdf, bool& specular,
                                                  float* eta_io = nullptr)
{
    specular = false;
    pdf = 0.0f;
    if (eta_io) *eta_io = 1.0f;
    const uint32_t n = m.n_layers;
    if (n == 0) return f3(0.0f, 0.0f, 0.0f);
    const uint32_t which = min((uint32_t)floorf(uc * (float)n), n - 1);
    const float3 wo = to_local(fr, wo_w);
    float3 wi;
    float3 f = layer_sample(m.layer[which], wo, u1, u2, wi, pdf);
    if (pdf == 0.0f) return f3(0.0f, 0.0f, 0.0f);
    wi_w = to_world(fr, wi);
    specular = kind_is_delta(layer_kind(m.layer[which]));
    if (eta_io && layer_kind(m.layer[which]) == kGlass) {
        const LayerDev& l = m.layer[which];
        *eta_io = wo.z > 0.0f ? l.q1.w / l.q2.w : l.q2.w / l.q1.w;
    }
    if (!specular) {
        for (uint32_t i = 0; i < n; i++)
            if (i != which && !kind_is_delta(layer_kind(m.layer[i]))) pdf += layer_pdf(m.layer[i], wi, wo);
        f = material_f(m, ng, wo_w, wi_w, wo, wi);
    }
    pdf /= (float)n;
    return f;
}

}  // namespace rb2dev
