/*
 * rb2_render.h -- camera rays and wavefront integrators on top of rb2.h.
 */
#ifndef RB2_RENDER_H
#define RB2_RENDER_H

#include "rb2.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Perspective camera.  Replaces PerspectiveCamera(position, lookat, up,
 * resolution, horizontal_fov) (core/camera.h:40-95): the host builds the
 * reference's raster->camera and camera->world matrices with the reference's
 * transform algebra (core/camera.cu:30-56), the device applies them exactly
 * as generate_ray does (core/camera.cu:91-98). */
typedef struct {
    float raster_to_camera[16];  /* row-major */
    float camera_to_world[16];   /* row-major */
    uint32_t width, height;
    float eye[3], lookat[3], up[3];
    float fov_deg;
} rb2_camera;

int rb2_camera_init(rb2_camera* cam, const float eye[3], const float lookat[3], const float up[3],
                    uint32_t width, uint32_t height, float fov_deg);

/* Writes width*height*spp camera rays (pixel-major: ray = pixel*spp + s) to
 * d_rays.  jitter == 0 samples pixel centres (x+0.5, y+0.5); otherwise the
 * offsets are PCG32 uniforms keyed by (seed, pixel, sample).  Pixel p is at
 * x = p % width, y = p / width (the reference's core/camera.h:73-75 swap of
 * width and height is not reproduced). */
int rb2_camera_rays(const rb2_camera* cam, uint32_t spp, uint64_t seed, int jitter, float* d_rays, void* stream);

/* Same for an explicit list of raster positions (2 floats each). */
int rb2_camera_rays_at(const rb2_camera* cam, const float* d_raster_xy, uint32_t n, float* d_rays, void* stream);

/* ------------------------------------------------------------- device scene --
 * Replaces Scene::gpu_prepare / SceneBuffer + MaterialBuffer
 * (core/scene.cpp:166-339, core/buffer.h:322-360) for the Lambertian +
 * diffuse-area-light subset the integrators use: per-material albedo and
 * emission (RGB); every triangle whose material emits is a light
 * (core/scene.cpp:105-113); lights are chosen uniformly per triangle. */
typedef struct rb2_scene_dev rb2_scene_dev;
int rb2_scene_create(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri,
                     const uint32_t* tri_material /* nullable: all 0 */, uint32_t n_materials,
                     const float* albedo_rgb /* nullable: 0.5 */, const float* emission_rgb /* nullable: 0 */,
                     rb2_scene_dev** out);
int rb2_scene_destroy(rb2_scene_dev* s);
int rb2_scene_device_bytes(const rb2_scene_dev* s, uint64_t* bytes);

/* Device view of a scene for the header-only rb2::trace_ray /
 * rb2::fill_intersection (rb2_device.cuh).  Replaces SceneBuffer
 * (core/buffer.h:322-345) for what the trace reads: vertex positions and
 * per-triangle vertex indices + material id. */
typedef struct {
    const void* verts;        /* float4 per vertex (xyz, w unused) */
    const void* tris;         /* uint4 per triangle (3 vertex indices, material id) */
    uint32_t nv, ntri;
} rb2_dev_scene;
int rb2_scene_dev_view(const rb2_scene_dev* s, rb2_dev_scene* out);

/* ------------------------------------------------------------- materials --
 * The reference's layered materials (core/material.h:44-51, at most 4
 * layers) over its BSDFs (core/reflection.cu): Lambertian, Oren-Nayar
 * (sigma in degrees, clamped to [0, 90]), specular mirror, specular
 * transmission ("glass": the reference's glass transmits only), and the
 * Torrance-Sparrow microfacet BSDF with a Blinn distribution and a
 * dielectric, conductor or no-op Fresnel term.  Scenes made by
 * rb2_scene_create use one Lambertian layer per material (albedo);
 * rb2_scene_set_materials replaces the layers of every material (emission is
 * kept; an emitter's layers are ignored).  Sampling follows
 * material_sample_f (core/material.cu:56-211) except that the combined pdf
 * of a multi-layer material is divided by the number of layers as in
 * pbrt-v2 (the reference left it undivided) and a glass layer adds no
 * microfacet term (a missing `break`, material.cu:204-209, Q11). */
enum {
    RB2_BSDF_LAMBERTIAN = 0, RB2_BSDF_OREN_NAYAR = 1, RB2_BSDF_MIRROR = 2, RB2_BSDF_GLASS = 3,
    RB2_BSDF_MICROFACET = 4, RB2_BSDF_EMITTER = 5
};
enum { RB2_FRESNEL_DIELECTRIC = 0, RB2_FRESNEL_CONDUCTOR = 1, RB2_FRESNEL_NOOP = 2 };
typedef struct {
    uint32_t type;          /* RB2_BSDF_LAMBERTIAN .. RB2_BSDF_MICROFACET */
    uint32_t fresnel;       /* microfacet: RB2_FRESNEL_* */
    float color[3];         /* reflectance (R of the microfacet BSDF) */
    float sigma_deg;        /* Oren-Nayar */
    float etai, etat;       /* glass; microfacet with a dielectric Fresnel */
    float exponent;         /* Blinn exponent */
    float eta[3], k[3];     /* microfacet with a conductor Fresnel */
} rb2_bsdf_layer;
typedef struct {
    uint32_t n_layers;      /* 1..4 (0 only for emitters) */
    uint32_t reserved;
    rb2_bsdf_layer layer[4];
} rb2_material_desc;
int rb2_scene_set_materials(rb2_scene_dev* s, const rb2_material_desc* materials, uint32_t n_materials);

/* Device evaluation of materials, for tests and tools: for query i with
 * material d_mat[i] and 9 floats d_q[9i..] = (n, wo, wi) in world space,
 * d_out[4i..] = (f rgb, pdf) of material_f / material_pdf with specular
 * layers excluded; with `sample` != 0, d_q holds (n, wo, u1, u2, uc) and
 * d_out[8i..] = (wi xyz, f rgb, pdf, 1 if a specular layer was sampled). */
int rb2_material_query(const rb2_scene_dev* s, int sample, const uint32_t* d_mat, const float* d_q, uint32_t n,
                       float* d_out, void* stream);

/* ------------------------------------------------------ intersection records --
 * Replaces CudaTracer::trace(const RayBuffer&, IntersectionBuffer&,
 * SceneBuffer&, uint8_t* stencil, bool any_hit) (cudatracer.h:87) with the
 * reference's SoA IntersectionBuffer (core/intersection.h:63-80), minus the
 * fields that trace leaves unwritten (tangent, bitangent, depth,
 * contribution).  Device pointers; any may be NULL to skip that field.
 * Closest hit fills every field of hit rays (kepler_dynamic_fetch.h:313-355)
 * and `intersected` of all rays; any hit writes `intersected` only; masked
 * rays get intersected = 0.  Shading normal = geometric normal (no vertex
 * normals), uv of the accepted triangle.  One persistent traversal launch
 * with the record written in the same kernel. */
typedef struct {
    float* position[3];
    float* geometric_normal[3];
    float* shading_normal[3];
    float* incoming_direction[3];
    float* uv;                      /* 2 floats per ray (float2) */
    uint32_t* primitive_id;
    uint32_t* primitive_material_id;
    uint8_t* front;
    uint8_t* intersected;
    float* epsilon;
} rb2_isect_buffer;
int rb2_trace_isect(rb2_tracer* t, const rb2_scene_dev* scene, const float* d_rays, uint32_t n, int any_hit,
                    const uint8_t* d_mask, const rb2_isect_buffer* out, void* stream);

/* ------------------------------------------------------------------- film --
 * Reconstruction filters of the reference's film (core/filter.h:46-132,
 * core/film.cpp:36-60, renderers/samplerrenderer.cu:103-168): a sample at
 * raster position (sx, sy) with radiance L adds w * L and w to every pixel
 * (x, y) with |x - (sx - 0.5)| <= xwidth and |y - (sy - 0.5)| <= ywidth, w
 * read from a 16 x 16 table of the filter evaluated at cell centres; a pixel's
 * value is max(0, sum(w L) / sum(w)).  Differences: the table is indexed by
 * x and y (the reference evaluated fx from the row index, core/film.cpp:56),
 * and each pixel gathers its samples in a fixed order instead of receiving
 * atomic adds, so images are deterministic.  RB2_FILTER_NONE is the
 * integrators' default: the mean of the pixel's own samples. */
enum { RB2_FILTER_NONE = 0, RB2_FILTER_BOX = 1, RB2_FILTER_TRIANGLE = 2, RB2_FILTER_GAUSSIAN = 3 };
typedef struct {
    uint32_t kind;          /* RB2_FILTER_* */
    float xwidth, ywidth;   /* half-widths in pixels, (0, 16] */
    float alpha;            /* Gaussian falloff (FilterGaussian's alpha) */
} rb2_filter;

/* Filter table exactly as the film precomputes it (16 x 16 floats, row y). */
int rb2_filter_table(const rb2_filter* f, float* table256);

/* Reconstructs an image from `spp` samples per pixel held sample-major
 * (sample j of pixel p at j * width * height + p): d_xy = raster positions
 * (2 floats; a sample of pixel p must lie in [px, px + 1) x [py, py + 1)),
 * d_L = radiance (4 floats, rgb + unused).  d_rgb: 3 floats per pixel. */
int rb2_film_develop(const rb2_filter* f, uint32_t width, uint32_t height, uint32_t spp, const float* d_xy,
                     const float* d_L, float* d_rgb, void* stream);

/* Portable float map (PFM, little-endian, bottom row first as the format
 * defines; rows of h_rgb are top first): the film's image file output. */
int rb2_image_write_pfm(const char* path, const float* h_rgb, uint32_t width, uint32_t height);

/* An integrator binds a tracer (BVH) and a device scene and owns the
 * wavefront scratch (grown on demand, reused across renders).  Replaces
 * Integrator::render(Scene*, CudaTracer*, void**, uint32_t) (core/integrator.h:59). */
typedef struct rb2_integrator rb2_integrator;
int rb2_integrator_create(rb2_tracer* tracer, const rb2_scene_dev* scene, rb2_integrator** out);
int rb2_integrator_destroy(rb2_integrator* it);
int rb2_integrator_device_bytes(const rb2_integrator* it, uint64_t* bytes);
/* Launch shape of the integrator's persistent traversals: block_threads 128
 * or 256, regs 64 or 48, fetch_threshold, node_threshold (zero fields: 128,
 * 24, a register budget of 48 for the binary layout and 64 for the compressed
 * 8-wide layout, a node-phase threshold of 8 for the binary layout and 16 for
 * the compressed one: the fastest shapes measured on configs 1-3;
 * ctas_per_sm is ignored).  Images do not depend on the shape. */
int rb2_integrator_set_launch(rb2_integrator* it, const rb2_launch_config* cfg);
/* Paths in flight per wave (0 = defaults: 32M paths for the path tracer,
 * 8M camera paths for BDPT).  The path tracer runs as many samples per pixel
 * at once as fit (unless rb2_pt_params.spp_per_wave is set); BDPT runs as many
 * iterations at once as fit, each with its own light-vertex cache.  Larger
 * waves mean larger traversal launches (less time in launch tails) and more
 * device memory.  Unfiltered images do not depend on the wave size. */
int rb2_integrator_set_wave(rb2_integrator* it, uint64_t paths);
/* Film filter of the path tracer, BDPT and ray casting (default RB2_FILTER_NONE); NULL resets. */
int rb2_integrator_set_filter(rb2_integrator* it, const rb2_filter* f);

/* Reference-compatibility switches (the `compat` fields below).  By default
 * the integrators correct four behaviours of the reference; each switch
 * reproduces one of them instead, so an image can be compared with what the
 * reference's own kernels would produce (in expectation: the random numbers
 * come from this library's generator, not thrust's).
 *  RB2_COMPAT_AO_DIRECTION  AO rays along X cos(phi) sin(theta) + Y sin(phi)
 *      sin(theta) + Z cos(phi), phi = 2 pi u1, theta = acos(sqrt(1 - u2)),
 *      about the unflipped geometric normal with the reference's choice of
 *      X and Y (core/montecarlo.cu:133-151): neither unit length nor
 *      cosine-distributed; tmax stays `radius` in units of that direction.
 *      Where X is undefined (a normal along +z or -z, whose cross product
 *      with the chosen axis vanishes) the reference's ray is NaN and never
 *      hits: the sample counts as unoccluded.
 *  RB2_COMPAT_RR_DIVISOR  Russian roulette from bounce rr_start + 1, and
 *      survivors divided by 1 - q instead of q (integrator_path.cu:232-244);
 *      needs rr_prob < 1.
 *  RB2_COMPAT_NEE_RESEED  next-event estimation draws the same light choice
 *      and point at every vertex of a path (the reference re-seeds its NEE
 *      generator each bounce, integrator_path.cu:113). */
enum { RB2_COMPAT_AO_DIRECTION = 1u << 0, RB2_COMPAT_RR_DIVISOR = 1u << 1, RB2_COMPAT_NEE_RESEED = 1u << 2 };

/* Ambient occlusion (AmbientOcclusionIntegratorParams, core/params.h:126-131;
 * integrators/integrator_ao.cu:42-110): one primary ray per pixel centre,
 * `samples` any-hit rays per hit from the hit point (tmin = 1e-3 t, tmax =
 * radius), cosine-distributed about the geometric normal facing the viewer.
 * d_ao[pixel] = unoccluded fraction (0 for pixels whose primary ray misses). */
typedef struct {
    uint32_t samples;
    float radius;
    uint64_t seed;
    uint32_t compat;         /* RB2_COMPAT_AO_DIRECTION or 0 */
    uint32_t reserved;
} rb2_ao_params;
int rb2_render_ao(rb2_integrator* it, const rb2_camera* cam, const rb2_ao_params* p, float* d_ao, void* stream);

/* Wavefront path tracing (PathIntegratorParams, core/params.h:88-94;
 * integrators/integrator_path.cu:43-283, the reference's declared
 * MODE_MULTI_KERNEL3).  Lambertian surfaces, or the scene's layered
 * materials (rb2_scene_set_materials; emission after a specular bounce takes
 * full weight), next-event estimation to a
 * uniformly chosen emissive triangle combined with BSDF sampling by the
 * balance heuristic, Russian roulette from bounce rr_start with continue
 * probability min(rr_prob, luminance(throughput)) and division by it.
 * Vertices 0..max_depth get NEE; extension rays are traced from vertices
 * below max_depth.  d_rgb[3*pixel] = mean radiance over spp jittered samples.
 * The reference's m_use_max_depth has no counterpart: its configuration code
 * reads it and none of its kernels use it, so max_depth always applies. */
typedef struct {
    uint32_t spp;
    uint32_t max_depth;
    uint32_t rr_start;
    float rr_prob;
    uint64_t seed;
    uint32_t spp_per_wave;   /* samples per pixel in flight at once (0 = auto) */
    uint32_t compat;         /* RB2_COMPAT_RR_DIVISOR | RB2_COMPAT_NEE_RESEED, or 0 */
} rb2_pt_params;
int rb2_render_pt(rb2_integrator* it, const rb2_camera* cam, const rb2_pt_params* p, float* d_rgb, void* stream);
/* Progressive path tracing: the checkpoint / resume form of rb2_render_pt for
 * long renders (the reference renders a whole frame at once and keeps no
 * render state, renderers/samplerrenderer.cu:182-196, MODE_PROGRESSIVE not
 * implemented in renderers/samplerrenderer.cpp:103-106).  Adds samples
 * [first_sample, first_sample + p->spp) of every pixel to the caller's running
 * sums d_sum (4 floats per pixel, 16-byte aligned: r, g, b sums, and the
 * filter weight sum when a film filter is set), zeroed by the caller before
 * the first call, and, when d_rgb is not NULL, writes the image over all
 * first_sample + p->spp samples summed so far.  Every call of one render
 * uses the same camera, seed, path parameters and film filter; only spp and
 * first_sample change.  A render can stop after any call and resume later
 * from a copy of d_sum and its sample count.  Without a
 * film filter, splitting the samples over calls gives the same bits as one
 * rb2_render_pt call of the total spp with the same seed; with one, the same
 * samples summed in another order (equal within float rounding). */
int rb2_render_pt_progressive(rb2_integrator* it, const rb2_camera* cam, const rb2_pt_params* p, uint32_t first_sample,
                              float* d_sum, float* d_rgb, void* stream);

/* Bidirectional path tracing with a light-vertex cache
 * (BidirectionalPathIntegratorLvcParams, core/params.h:103-118;
 * integrators/integrator_bdpt_lvc_sk.cu:47-514).  Per iteration (one camera
 * sample per pixel): num_light_paths light subpaths are traced and every
 * surface vertex is stored in the cache (slots assigned by a prefix scan over
 * (path, depth), so the cache is deterministic); each camera vertex then adds
 * emission (s = 0), next-event estimation (s = 1) and `connections`
 * connections to uniformly chosen cached vertices (s >= 2, scaled by
 * cached vertices / light paths).  A path of k segments (k <= max_path_length)
 * is sampled by emission and by a connection across each edge whose two
 * endpoints scatter non-specularly on that path (the camera counts as
 * specular, the light point as non-specular); each of those n strategies is
 * weighted 1/n, which is 1/k when no vertex is specular, so the estimator is
 * unbiased.  (The reference weights connections by 1/((bounce+1)+depth) but
 * gives NEE full weight and omits the cache-size factor.)  Layered materials,
 * mirror and glass layers included: vertices take f from the material
 * functions (a connection uses the non-specular part), vertices of purely
 * specular materials are not cached, light subpaths continue with the adjoint
 * f(sampled -> incoming) because the Blinn microfacet's shadowing term is not
 * symmetric, and a glass transmission sampled on a light subpath takes the
 * adjoint factor (eta of the outgoing side / eta of the incoming side)^6 times
 * the camera-side factor.  d_rgb[3*pixel] = mean radiance over spp iterations. */
/* The reference's BidirectionalPathIntegratorLvcParams (core/params.h:108-120)
 * map as follows: m_num_light_paths -> num_light_paths;
 * m_num_cam_path_connections (sample_N) -> connections; m_cam_path_rrstart and
 * m_light_path_rrstart -> rr_start, one value for both subpaths (the
 * reference's own integrator file gives both the same value);
 * m_cam_path_rrprob -> rr_prob; m_num_cam_path_max_depth and
 * m_num_light_path_max_depth -> max_path_length, one cap on the whole path
 * (light subpaths keep at most max_path_length - 2 surface vertices).  No
 * field replaces m_num_prep_paths: the cache is sized exactly by a prefix scan,
 * so no preparation pass runs.  m_num_cam_path_sample_connections (sample_M)
 * is read by the reference's configuration code but used by none of its
 * kernels.  m_mode (sk, mk, sort) has no counterpart: the three reference
 * kernels compute one estimator, which this wavefront implementation runs. */
typedef struct {
    uint32_t spp;
    uint32_t max_path_length;   /* segments, camera to light (config 3: 6) */
    uint32_t num_light_paths;   /* per iteration (0 = one per pixel) */
    uint32_t connections;       /* cached vertices per camera vertex (1..8) */
    uint32_t rr_start;
    float rr_prob;
    uint64_t seed;
} rb2_bdpt_params;
int rb2_render_bdpt(rb2_integrator* it, const rb2_camera* cam, const rb2_bdpt_params* p, float* d_rgb, void* stream);

/* The reference's full BidirectionalPathIntegratorLvcParams (core/params.h:108-120,
 * read from its integrator file by config/configuration.cpp:251-300), plus
 * the estimator choice.
 *
 * RB2_BDPT_ESTIMATOR_UNBIASED: the estimator of rb2_render_bdpt above, with
 *   max_path_length the whole-path cap, light_path_rrstart and
 *   cam_path_rrstart the bounces from which each subpath plays Russian
 *   roulette (continue probability min(cam_path_rrprob, luminance)), and the
 *   two max-depth fields unused (the whole-path cap bounds both subpaths).
 * RB2_BDPT_ESTIMATOR_REFERENCE: the reference's own estimator
 *   (integrators/integrator_bdpt_lvc_sk.cu:47-514), field for field:
 *   - a preparation pass of num_prep_paths light subpaths sizes the cache at
 *     ceil(1.1 * mean stored vertices per path * num_light_paths) vertices;
 *     a light subpath stops storing once the cache is full (the cache keeps
 *     the first vertices in (path, depth) order);
 *   - light subpaths start as DiffuseAreaLight::Le does (core/lights.cu:63-69):
 *     a direction drawn uniformly from the hemisphere about world +z and
 *     negated, contribution Le / pdf with no factor for the choice of
 *     emissive triangle; they store every surface vertex they hit and play
 *     roulette at every bounce with continue probability
 *     min(1, luminance(f |cos| / pdf)), and stop when their contribution is
 *     black.  The reference never caps their length; here they keep at most
 *     num_light_path_max_depth vertices (its integrator file: 8), which bounds
 *     the cache;
 *   - camera vertices 0..num_cam_path_max_depth add emission (first vertex or
 *     after a specular bounce, full weight), next-event estimation at full
 *     weight with the same draws at every vertex (the reference re-seeds each
 *     bounce), and num_cam_path_connections connections to uniformly chosen
 *     cached vertices, each weighted 1 / ((bounce + 1) + depth of the cached
 *     vertex) with no cache-size factor;
 *   - camera Russian roulette from bounce cam_path_rrstart + 1 with continue
 *     probability min(cam_path_rrprob, luminance) and survivors divided by
 *     1 - that probability (needs cam_path_rrprob < 1);
 *   - light_path_rrstart and num_cam_path_sample_connections are accepted and,
 *     as in the reference's kernels, not used; mode (sk, mk, sort) selects
 *     among three kernel organisations of one estimator there, and this
 *     wavefront implementation runs that estimator for each.
 *   The light point of a subpath starts 1e-4 off the light (the reference's
 *   ray starts on it and can hit its own light at a rounding-level t). */
enum { RB2_BDPT_ESTIMATOR_UNBIASED = 0, RB2_BDPT_ESTIMATOR_REFERENCE = 1 };
enum { RB2_BDPT_MODE_SK = 0, RB2_BDPT_MODE_MK = 1, RB2_BDPT_MODE_SORT = 2 };
typedef struct {
    uint32_t spp;                              /* iterations (one camera sample per pixel each) */
    uint32_t num_prep_paths;                   /* m_num_prep_paths (reference estimator; 0 = no cap) */
    uint32_t num_light_paths;                  /* m_num_light_paths per iteration (0 = one per pixel) */
    uint32_t num_light_path_max_depth;         /* m_num_light_path_max_depth (reference estimator) */
    uint32_t light_path_rrstart;               /* m_light_path_rrstart */
    uint32_t num_cam_path_max_depth;           /* m_num_cam_path_max_depth (reference estimator) */
    uint32_t cam_path_rrstart;                 /* m_cam_path_rrstart */
    float cam_path_rrprob;                     /* m_cam_path_rrprob */
    uint32_t num_cam_path_sample_connections;  /* m_num_cam_path_sample_connections (sample_M) */
    uint32_t num_cam_path_connections;         /* m_num_cam_path_connections (sample_N), 1..8 */
    uint32_t mode;                             /* m_mode: RB2_BDPT_MODE_* */
    uint32_t estimator;                        /* RB2_BDPT_ESTIMATOR_* */
    uint32_t max_path_length;                  /* unbiased estimator: segments camera to light, 1..16 */
    uint32_t reserved;
    uint64_t seed;
} rb2_bdpt_lvc_params;
int rb2_render_bdpt_lvc(rb2_integrator* it, const rb2_camera* cam, const rb2_bdpt_lvc_params* p, float* d_rgb,
                        void* stream);

/* Ray casting (RayCastIntegratorParams / RayCastShade, core/params.h:139-151;
 * IntegratorRayCast::compute and kernel_ray_cast_update,
 * integrators/integrator_raycast.cu:27-113): spp jittered camera samples per
 * pixel (the path tracer's sample positions for the same seed), one
 * closest-hit traversal, one colour per sample from its hit:
 *   PRIMITIVE_ID  the reference's 15-entry palette at (primitive id mod 15);
 *   MATERIAL_ID   the colour of the hit material's first layer (Lambertian,
 *                 mirror, glass, microfacet R; the emission of an emitter;
 *                 black for Oren-Nayar, which the reference does not handle);
 *   NORMALS       the shading normal, which is the unflipped geometric normal
 *                 normalize(cross(v1 - v0, v2 - v0)) for these scenes;
 *   UVS           black (the reference leaves this mode empty);
 *   UNIFORM       1 on a hit.
 * Misses are black.  d_rgb[3*pixel] = mean over the samples, or the filtered
 * value when a film filter is set (rb2_integrator_set_filter). */
enum {
    RB2_RAYCAST_SHADE_PRIMITIVE_ID = 0,
    RB2_RAYCAST_SHADE_MATERIAL_ID = 1,
    RB2_RAYCAST_SHADE_NORMALS = 2,
    RB2_RAYCAST_SHADE_UVS = 3,
    RB2_RAYCAST_SHADE_UNIFORM = 4
};
typedef struct {
    uint32_t spp;
    uint32_t shade;   /* RB2_RAYCAST_SHADE_* */
    uint64_t seed;
} rb2_raycast_params;
int rb2_render_raycast(rb2_integrator* it, const rb2_camera* cam, const rb2_raycast_params* p, float* d_rgb,
                       void* stream);

/* Statistics of the last render on this integrator (rays traced per kind);
 * trace_ms = GPU time of its traversal launches (CUDA events around each),
 * measured only while rb2_integrator_set_timing(it, 1) is on, else 0. */
typedef struct {
    uint64_t primary_rays, extension_rays, shadow_rays, connection_rays, light_rays;
    uint64_t lvc_vertices;
    double trace_ms;
} rb2_render_stats;
int rb2_integrator_set_timing(rb2_integrator* it, int on);
int rb2_integrator_stats(rb2_integrator* it, rb2_render_stats* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
