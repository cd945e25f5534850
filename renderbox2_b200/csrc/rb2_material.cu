// Layered materials: host packing (rb2_scene_set_materials) and the device
// query entry used by the tests (rb2_material_query).
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_internal.h"
#include "rb2_material.cuh"
#include "rb2_render.h"
#include "rb2_render_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace rb2dev {

__global__ void k_material_query(const MaterialDev* mats, uint32_t n_mat, int sample, const uint32_t* mat,
                                 const float* q, uint32_t n, float* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MaterialDev& m = mats[min(mat[i], n_mat - 1)];
        const float* qi = q + 9 * (size_t)i;
        const float3 ng = f3(qi[0], qi[1], qi[2]), wo_w = f3(qi[3], qi[4], qi[5]);
        const Frame fr = frame_from_z(ng);
        if (sample) {
            float3 wi_w = f3(0.0f, 0.0f, 0.0f);
            float pdf;
            bool spec;
            const float3 f = material_sample(m, fr, ng, wo_w, qi[6], qi[7], qi[8], wi_w, pdf, spec);
            float* o = out + 8 * (size_t)i;
            o[0] = wi_w.x; o[1] = wi_w.y; o[2] = wi_w.z; o[3] = f.x; o[4] = f.y; o[5] = f.z; o[6] = pdf;
            o[7] = spec ? 1.0f : 0.0f;
        } else {
            const float3 wi_w = f3(qi[6], qi[7], qi[8]);
            const float3 wo = to_local(fr, wo_w), wi = to_local(fr, wi_w);
            const float3 f = material_f(m, ng, wo_w, wi_w, wo, wi);
            float* o = out + 4 * (size_t)i;
            o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = material_pdf(m, wo, wi);
        }
    }
}

}  // namespace rb2dev

using namespace rb2;

namespace {

int cuda_fail(cudaError_t e, const char* what) { return fail(rb2::cuda_status(e), std::string(what) + ": " + cudaGetErrorString(e)); }

// One layer in the device packing; Oren-Nayar A, B as the scene reader
// computes them (io/customfilereader.cpp:128-136).
int pack_layer(const rb2_bsdf_layer& l, rb2dev::LayerDev& d)
{
    if (l.type > RB2_BSDF_MICROFACET) return fail(RB2_EINVAL, "unknown bsdf layer type");
    if (l.type == RB2_BSDF_MICROFACET && l.fresnel > RB2_FRESNEL_NOOP) return fail(RB2_EINVAL, "unknown Fresnel type");
    if ((l.type == RB2_BSDF_GLASS || (l.type == RB2_BSDF_MICROFACET && l.fresnel == RB2_FRESNEL_DIELECTRIC)) &&
        !(l.etai > 0.0f && l.etat > 0.0f))
        return fail(RB2_EINVAL, "indices of refraction must be positive");
    if (l.type == RB2_BSDF_MICROFACET && !(l.exponent >= 0.0f && std::isfinite(l.exponent)))
        return fail(RB2_EINVAL, "Blinn exponent must be >= 0");
    float A = 1.0f, B = 0.0f;
    if (l.type == RB2_BSDF_OREN_NAYAR) {
        const float sigma = std::min(std::max(l.sigma_deg, 0.0f), 90.0f) * (3.14159265358979323846f / 180.0f);
        const float s2 = sigma * sigma;
        A = 1.0f - (s2 / (2.0f * (s2 + 0.33f)));
        B = 0.45f * s2 / (s2 + 0.09f);
    }
    uint32_t kind = l.type, fres = l.fresnel;
    float qz, qw;
    std::memcpy(&qz, &kind, 4);
    std::memcpy(&qw, &fres, 4);
    d.q0 = make_float4(l.color[0], l.color[1], l.color[2], l.exponent);
    d.q1 = make_float4(l.eta[0], l.eta[1], l.eta[2], l.etai);
    d.q2 = make_float4(l.k[0], l.k[1], l.k[2], l.etat);
    d.q3 = make_float4(A, B, qz, qw);
    return RB2_OK;
}

}  // namespace

extern "C" {

int rb2_scene_set_materials(rb2_scene_dev* s, const rb2_material_desc* materials, uint32_t n_materials)
{
    if (!s || (n_materials && !materials)) return fail(RB2_EINVAL, "null argument");
    if (n_materials != s->n_mat) return fail(RB2_EINVAL, "one description per scene material is required");
    std::vector<float4> emi(s->n_mat), alb(s->n_mat);
    cudaError_t e;
    if ((e = cudaMemcpy(emi.data(), s->d_emission, s->n_mat * sizeof(float4), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "emission read");
    if ((e = cudaMemcpy(alb.data(), s->d_albedo, s->n_mat * sizeof(float4), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "albedo read");
    std::vector<rb2dev::MaterialDev> mats(s->n_mat);
    bool layered = false;
    for (uint32_t m = 0; m < s->n_mat; m++) {
        const rb2_material_desc& d = materials[m];
        rb2dev::MaterialDev& md = mats[m];
        std::memset(&md, 0, sizeof(md));
        const bool emitter = emi[m].x > 0.0f || emi[m].y > 0.0f || emi[m].z > 0.0f;
        if (emitter) continue;  // emitters end paths; their layers are not used
        if (d.n_layers < 1 || d.n_layers > rb2dev::kMaxLayers) return fail(RB2_EINVAL, "materials have 1 to 4 layers");
        md.n_layers = d.n_layers;
        bool nondelta = false;
        for (uint32_t i = 0; i < d.n_layers; i++) {
            int rc = pack_layer(d.layer[i], md.layer[i]);
            if (rc) return rc;
            nondelta |= d.layer[i].type != RB2_BSDF_MIRROR && d.layer[i].type != RB2_BSDF_GLASS;
        }
        const bool plain = d.n_layers == 1 && d.layer[0].type == RB2_BSDF_LAMBERTIAN;
        md.flags = (plain ? rb2dev::kMatPlainLambertian : 0u) | (nondelta ? rb2dev::kMatHasNonDelta : 0u);
        if (plain) alb[m] = make_float4(d.layer[0].color[0], d.layer[0].color[1], d.layer[0].color[2], 0.0f);
        layered |= !plain;
    }
    rb2dev::MaterialDev* dm = nullptr;
    if ((e = rb2::dev_malloc(&dm, mats.size() * sizeof(rb2dev::MaterialDev))) != cudaSuccess)
        return fail(RB2_ENOMEM, std::string("material table: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpy(dm, mats.data(), mats.size() * sizeof(rb2dev::MaterialDev), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_albedo, alb.data(), s->n_mat * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess) {
        rb2::dev_free(dm);
        return cuda_fail(e, "material upload");
    }
    if (s->d_mats) {
        s->bytes -= (uint64_t)s->n_mat * sizeof(rb2dev::MaterialDev);
        rb2::dev_free(s->d_mats);
    }
    s->d_mats = dm;
    s->layered = layered;
    s->bytes += (uint64_t)s->n_mat * sizeof(rb2dev::MaterialDev);
    return RB2_OK;
}

int rb2_material_query(const rb2_scene_dev* s, int sample, const uint32_t* d_mat, const float* d_q, uint32_t n,
                       float* d_out, void* stream)
{
    if (!s || (n && (!d_mat || !d_q || !d_out))) return fail(RB2_EINVAL, "null argument");
    if (!s->d_mats) return fail(RB2_EINVAL, "scene has no material table (rb2_scene_set_materials)");
    if (n == 0) return RB2_OK;
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, 4096);
    rb2dev::k_material_query<<<g, 256, 0, (cudaStream_t)stream>>>(s->d_mats, s->n_mat, sample, d_mat, d_q, n, d_out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RB2_OK : cuda_fail(e, "material query launch");
}

}  // extern "C"
