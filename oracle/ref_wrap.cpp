// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C entry points over the reference's own host code, compiled in place from
// the reference sources (see oracle/Makefile).  The reference SBVH builder
// (accelerators/sbvh/splitbvhbuilder.cpp:177-214, 234-626) and Compact2 packer
// (accelerators/sbvh/cudabvh.cpp:216-322) run exactly as written; this file
// only feeds them a Scene and copies their buffers out through plain pointers.
// It also exposes the reference's text BVH cache (cudabvh.cpp:108-214), its
// perspective camera (core/camera.cu:30-98) and its host Moller-Trumbore test
// (core/primitives.cu:51-70) so the CPU restatement and the product can be
// pinned against them, and its BSDFs and material dispatch
// (core/reflection.cu, core/material.cu) for the BSDF pin.
#include <accelerators/sbvh/bvh.h>
#include <accelerators/sbvh/cudabvh.h>
#include <core/bsdf.h>
#include <core/util.h>
#include <core/camera.h>
#include <core/lights.h>
#include <core/montecarlo.h>
#include <core/material.h>
#include <core/mesh.h>
#include <core/primitives.h>
#include <core/scene.h>
#include <memory/memoryallocator.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

using namespace renderbox2;

extern "C" {

struct rb2ref_bvh {
    uint32_t n_nodes;    // uint4 count
    uint32_t n_woop;     // uint4 count
    uint32_t n_triidx;   // uint32 count
    uint32_t layout;
    uint32_t* nodes;     // 4*n_nodes words
    uint32_t* woop;      // 4*n_woop words
    uint32_t* triidx;    // n_triidx words
    float sah;
    uint32_t n_inner, n_leaves, n_tri_refs;
    double build_ms;
};

void rb2ref_free(rb2ref_bvh* b)
{
    if (!b) return;
    std::free(b->nodes);
    std::free(b->woop);
    std::free(b->triidx);
    b->nodes = b->woop = nullptr;
    b->triidx = nullptr;
}

}  // extern "C"

namespace {

struct StdoutSilencer {
    int saved = -1;
    explicit StdoutSilencer(bool on)
    {
        if (!on) return;
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }
    ~StdoutSilencer()
    {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

// The reference Scene's destructor frees device buffers it never allocated
// unless gpu_prepare() ran, so scenes made here are intentionally leaked.
Scene* make_scene(const float* v, uint32_t nv, const uint32_t* idx, uint32_t ntri)
{
    static MemoryAllocator* alloc = new MemoryAllocator();
    Scene* scene = new Scene(*alloc);
    Mesh m;
    m.m_name = "oracle";
    for (uint32_t i = 0; i < nv; i++) {
        float3 p = make_float3(v[3 * i + 0], v[3 * i + 1], v[3 * i + 2]);
        m.m_vertices.push_back(p);
        m.m_bounds.insert(p);
    }
    for (uint32_t t = 0; t < ntri; t++) {
        m.m_vtx_indices.push_back(make_uint3(idx[3 * t + 0], idx[3 * t + 1], idx[3 * t + 2]));
        m.m_nor_indices.push_back(make_uint3(0, 0, 0));
        m.m_mat_ids.push_back(0);
    }
    scene->add_mesh(m, false);
    return scene;
}

void copy_out(const CudaBvh& cb, rb2ref_bvh* out)
{
    const auto& n = cb.get_node_buffer();
    const auto& w = cb.get_tri_woop_buffer();
    const auto& t = cb.get_tri_index_buffer();
    out->n_nodes = (uint32_t)n.size();
    out->n_woop = (uint32_t)w.size();
    out->n_triidx = (uint32_t)t.size();
    out->layout = (uint32_t)cb.get_layout();
    out->nodes = (uint32_t*)std::malloc(sizeof(uint4) * (n.size() + 1));
    out->woop = (uint32_t*)std::malloc(sizeof(uint4) * (w.size() + 1));
    out->triidx = (uint32_t*)std::malloc(sizeof(uint32_t) * (t.size() + 1));
    std::memcpy(out->nodes, n.data(), sizeof(uint4) * n.size());
    std::memcpy(out->woop, w.data(), sizeof(uint4) * w.size());
    std::memcpy(out->triidx, t.data(), sizeof(uint32_t) * t.size());
}

}  // namespace

extern "C" {

// Builds the reference SBVH over (v, idx) with the default Platform and
// BuildParams and packs it as BVHLayout_Compact2 (the Kepler layout the
// reference selects, core/application.cpp:121-127).  Optionally writes the
// reference's text cache to `cache_path`.  Returns 0 on success.
int rb2ref_build(const float* v, uint32_t nv, const uint32_t* idx, uint32_t ntri, int quiet,
                 const char* cache_path, rb2ref_bvh* out)
{
    if (!v || !idx || !out || ntri == 0) return -1;
    std::memset(out, 0, sizeof(*out));
    StdoutSilencer silence(quiet != 0);
    Scene* scene = make_scene(v, nv, idx, ntri);
    Platform platform;
    BVH::Stats stats;
    BVH::BuildParams params;
    params.m_enable_prints = false;
    params.m_stats = &stats;
    auto t0 = std::chrono::steady_clock::now();
    BVH bvh(scene, platform, params);
    CudaBvh cb(bvh, BVHLayout::BVHLayout_Compact2);
    auto t1 = std::chrono::steady_clock::now();
    out->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    out->sah = stats.m_sah_cost;
    out->n_inner = stats.m_num_inner_nodes;
    out->n_leaves = stats.m_num_leaf_nodes;
    out->n_tri_refs = stats.m_num_tris;
    copy_out(cb, out);
    if (cache_path && cache_path[0]) cb.serialize(std::string(cache_path));
    return 0;
}

// Loads a reference text cache through CudaBvh(const std::string&, bool&).
int rb2ref_load(const char* path, rb2ref_bvh* out)
{
    if (!path || !out) return -1;
    std::memset(out, 0, sizeof(*out));
    bool ok = false;
    CudaBvh cb{std::string(path), ok};
    if (!ok) return -2;
    copy_out(cb, out);
    return 0;
}

// PerspectiveCamera(eye, lookat, up, (w,h), fov).generate_ray(x, y) for n
// raster positions; writes 8 floats per ray (origin, tmin, dir, tmax).
int rb2ref_camera_rays(const float* eye, const float* look, const float* up, float w, float h, float fov,
                       const float* raster_xy, uint32_t n, float* rays_out)
{
    PerspectiveCamera cam(make_float3(eye[0], eye[1], eye[2]), make_float3(look[0], look[1], look[2]),
                          make_float3(up[0], up[1], up[2]), make_float2(w, h), fov);
    for (uint32_t i = 0; i < n; i++) {
        Ray r = cam.generate_ray(raster_xy[2 * i + 0], raster_xy[2 * i + 1]);
        float3 o = r.origin(), d = r.direction();
        float* dst = rays_out + 8 * (size_t)i;
        dst[0] = o.x; dst[1] = o.y; dst[2] = o.z; dst[3] = r.tmin();
        dst[4] = d.x; dst[5] = d.y; dst[6] = d.z; dst[7] = r.tmax();
    }
    return 0;
}

// Host Moller-Trumbore from the reference; returns 1 on hit and (u, v, t).
int rb2ref_intersect_triangle(const float* v0, const float* v1, const float* v2, const float* ray8, float* uvt)
{
    Ray r(make_float4(ray8[0], ray8[1], ray8[2], ray8[3]), make_float4(ray8[4], ray8[5], ray8[6], ray8[7]));
    float3 res;
    bool hit = intersect_ray_triangle(make_float3(v0[0], v0[1], v0[2]), make_float3(v1[0], v1[1], v1[2]),
                                      make_float3(v2[0], v2[1], v2[2]), r, res);
    uvt[0] = res.x; uvt[1] = res.y; uvt[2] = res.z;
    return hit ? 1 : 0;
}

// compute_normal (core/primitives.h:267-270) and Ray::operator() (:171-174)
// from the reference, for pinning the intersection-record arithmetic.
int rb2ref_normal_and_point(const float* v0, const float* v1, const float* v2, const float* ray8, float t,
                            float* ng_out, float* p_out)
{
    float3 n = compute_normal(make_float3(v0[0], v0[1], v0[2]), make_float3(v1[0], v1[1], v1[2]),
                              make_float3(v2[0], v2[1], v2[2]));
    Ray r(make_float4(ray8[0], ray8[1], ray8[2], ray8[3]), make_float4(ray8[4], ray8[5], ray8[6], ray8[7]));
    float3 p = r(t);
    ng_out[0] = n.x; ng_out[1] = n.y; ng_out[2] = n.z;
    p_out[0] = p.x; p_out[1] = p.y; p_out[2] = p.z;
    return 0;
}

// One bxdf layer in the product's rb2_bsdf_layer layout (60 bytes).
struct rb2ref_layer {
    uint32_t type, fresnel;
    float color[3], sigma_deg, etai, etat, exponent, eta[3], k[3];
};

// The reference's material_f + material_pdf (sample == 0; q = n, wo, wi) or
// material_sample_f (sample != 0; q = n, wo, u1, u2, uc) for one material
// built as the scene reader builds it (io/customfilereader.cpp:99-211):
// per-type parameter arrays, bxdf type bits, Oren-Nayar A, B from sigma.
// Non-specular queries use flags BxDF_ALL & ~BxDF_SPECULAR, sampling BxDF_ALL,
// as the path integrator calls them (integrators/integrator_path.cu:150-222).
// out = (f rgb, pdf) or (wi xyz, f rgb, pdf, specular).
int rb2ref_material(const rb2ref_layer* layers, uint32_t n_layers, int sample, const float* q, float* out)
{
    if (n_layers == 0 || n_layers > 4) return 1;
    Material m{};
    LambertianBsdfParams lam[4];
    OrenNayarBsdfParams on[4];
    MirrorBsdfParams mir[4];
    GlassBsdfParams gl[4];
    MicrofacetBsdfParams mf[4];
    uint32_t nl = 0, non = 0, nm = 0, ng = 0, nmf = 0;
    for (uint32_t i = 0; i < n_layers; i++) {
        const rb2ref_layer& L = layers[i];
        const float4 color = make_float4(L.color[0], L.color[1], L.color[2], 0.0f);
        switch (L.type) {
        case 0:
            m.layer_bxdf_type[i] = BxDFType(BxDF_REFLECTION | BxDF_DIFFUSE);
            m.layer_bsdf_type[i] = BSDF_LAMBERTIAN;
            m.layer_bsdf_id[i] = nl;
            lam[nl++].color = color;
            break;
        case 1: {
            m.layer_bxdf_type[i] = BxDFType(BxDF_REFLECTION | BxDF_DIFFUSE);
            m.layer_bsdf_type[i] = BSDF_OREN_NAYAR;
            m.layer_bsdf_id[i] = non;
            OrenNayarBsdfParams& p = on[non++];
            p.color = color;
            p.sigma = to_radians(clamp(L.sigma_deg, 0.0f, 90.0f));
            const float s2 = p.sigma * p.sigma;
            p.AB.x = 1.0f - (s2 / (2.0f * (s2 + 0.33f)));
            p.AB.y = 0.45f * s2 / (s2 + 0.09f);
            break;
        }
        case 2:
            m.layer_bxdf_type[i] = BxDFType(BxDF_REFLECTION | BxDF_SPECULAR);
            m.layer_bsdf_type[i] = BSDF_MIRROR;
            m.layer_bsdf_id[i] = nm;
            mir[nm++].color = color;
            break;
        case 3:
            m.layer_bxdf_type[i] = BxDFType(BxDF_REFLECTION | BxDF_SPECULAR | BxDF_TRANSMISSION);
            m.layer_bsdf_type[i] = BSDF_GLASS;
            m.layer_bsdf_id[i] = ng;
            gl[ng].color = color;
            gl[ng].etai = L.etai;
            gl[ng++].etat = L.etat;
            break;
        case 4: {
            m.layer_bxdf_type[i] = BxDFType(BxDF_REFLECTION | BxDF_GLOSSY);
            m.layer_bsdf_type[i] = BSDF_BLINN_MICROFACET;
            m.layer_bsdf_id[i] = nmf;
            MicrofacetBsdfParams& p = mf[nmf++];
            p.R = color;
            p.exponent = L.exponent;
            p.type = L.fresnel == 1 ? FresnelType::FRESNEL_CONDUCTOR
                                    : (L.fresnel == 0 ? FresnelType::FRESNEL_DIELECTRIC : FresnelType::FRESNEL_NOOP);
            p.eta = make_float4(L.eta[0], L.eta[1], L.eta[2], 0.0f);
            p.k = make_float4(L.k[0], L.k[1], L.k[2], 0.0f);
            p.etai = L.etai;
            p.etat = L.etat;
            break;
        }
        default:
            return 1;
        }
    }
    m.num_valid_layers = n_layers;
    m.m_emitter = 0;
    MaterialBuffer mb{};
    mb.m_materials = &m;
    mb.m_lambertian_bsdfs = lam;
    mb.m_orennayar_bsdfs = on;
    mb.m_mirror_bsdfs = mir;
    mb.m_glass_bsdfs = gl;
    mb.m_microfacet_bsdfs = mf;
    mb.m_num_materials = 1;
    const float3 n = make_float3(q[0], q[1], q[2]);
    const float3 wo = make_float3(q[3], q[4], q[5]);
    Frame frame;
    frame.set_from_z(n);
    if (sample) {
        BsdfSample bs;
        bs.m_dir1 = q[6];
        bs.m_dir2 = q[7];
        bs.fComponent = q[8];
        bs.pad = 0.0f;
        float3 wi = make_float3(0.0f);
        float pdf = 0.0f;
        BxDFType st = BxDFType(0);
        const float3 f = material_sample_f(mb, 0, wo, frame, n, bs, wi, pdf, BxDF_ALL, st);
        out[0] = wi.x; out[1] = wi.y; out[2] = wi.z;
        out[3] = f.x; out[4] = f.y; out[5] = f.z; out[6] = pdf;
        out[7] = (st & BxDF_SPECULAR) ? 1.0f : 0.0f;
    } else {
        const float3 wi = make_float3(q[6], q[7], q[8]);
        const BxDFType fl = BxDFType(BxDF_ALL & ~BxDF_SPECULAR);
        const float3 f = material_f(mb, 0, wo, wi, n, frame, fl);
        out[0] = f.x; out[1] = f.y; out[2] = f.z;
        out[3] = material_pdf(mb, 0, wo, wi, frame, fl);
    }
    return 0;
}

// cosine_sample_hemisphere_normal (core/montecarlo.cu:133-151), the
// reference's AO direction about `normal`.
int rb2ref_ao_direction(float u1, float u2, const float* normal, float* dir_out)
{
    float3 n = make_float3(normal[0], normal[1], normal[2]);
    float3 d = cosine_sample_hemisphere_normal(u1, u2, n);
    dir_out[0] = d.x; dir_out[1] = d.y; dir_out[2] = d.z;
    return 0;
}

// DiffuseAreaLight(v0, v1, v2, emit).Le(...) (core/lights.cu:63-69): writes
// the light point, the direction, the pdf and the returned radiance.
int rb2ref_light_le(const float* v0, const float* v1, const float* v2, const float* emit, const float* u5,
                    float* pt_out, float* dir_out, float* pdf_out, float* L_out)
{
    DiffuseAreaLight l(make_float3(v0[0], v0[1], v0[2]), make_float3(v1[0], v1[1], v1[2]),
                       make_float3(v2[0], v2[1], v2[2]), make_float3(emit[0], emit[1], emit[2]));
    LightSample sample;
    sample.m_u0 = u5[0];
    sample.m_u1 = u5[1];
    float3 pt, dir;
    float pdf = 0.0f;
    float3 L = l.Le(sample, make_float2(u5[2], u5[3]), pt, dir, pdf);
    pt_out[0] = pt.x; pt_out[1] = pt.y; pt_out[2] = pt.z;
    dir_out[0] = dir.x; dir_out[1] = dir.y; dir_out[2] = dir.z;
    *pdf_out = pdf;
    L_out[0] = L.x; L_out[1] = L.y; L_out[2] = L.z;
    return 0;
}

}  // extern "C"
