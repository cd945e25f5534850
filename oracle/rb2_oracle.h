/*
 * TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's ray traversal,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The product library never includes, links or calls this.
 *
 * Parity pin: the traversal is restated from the reference's single-ray
 * trace_ray (accelerators/sbvh/cuda_tracer_functions.cu:42-279) and its span
 * helpers (accelerators/sbvh/cudatracerkernels.h:213-256).  The reference
 * ships no tests or golden vectors, so this restatement is pinned against the
 * reference's own host code compiled in place (oracle/_ref: SBVH builder,
 * Compact2 packer, camera, Moller-Trumbore) and against committed fixtures
 * generated from it (tests/golden/).
 */
#ifndef RB2_ORACLE_H
#define RB2_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int32_t prim; float t, u, v; } rb2o_hit;
typedef struct { uint32_t nodes, tris, leafterms, pad; } rb2o_counts;

/* Closest-hit / any-hit over Compact2 buffers (4 words per uint4).
 * rays: 8 floats per ray (ox, oy, oz, tmin, dx, dy, dz, tmax).
 * mask (nullable): rays with mask[i]==0 are skipped and report prim=-1.
 * counts (nullable): canonical single-lane visit counts per ray.
 * nthreads <= 0: use all OpenMP threads. */
void rb2o_trace(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx,
                const float* rays, uint32_t n, int any_hit, const uint8_t* mask,
                rb2o_hit* out, rb2o_counts* counts, int nthreads);

/* Single Woop triangle test with the same arithmetic as the traversal.
 * Returns 1 and (t,u,v) when tmin < t < tmax and the barycentrics pass. */
int rb2o_woop_test(const uint32_t* woop12, const float* ray8, float tmax, float* tuv);

/* Brute force over every Woop triangle slot (closest accepted t; on equal t
 * the first slot wins).  Returns hit records with the original triangle id. */
void rb2o_bruteforce(const uint32_t* woop, const uint32_t* triidx, uint32_t n_woop_u4,
                     const float* rays, uint32_t n, rb2o_hit* out, int nthreads);

/* Tie count per ray: the number of distinct triangles whose Woop test
 * accepts the ray at exactly its closest-hit t (hits[i].t; 0 for misses).
 * A ray through a shared edge or vertex of triangles that agree on t counts
 * 2 or more.  _brute tests every Woop slot (exact; small scenes); the other
 * walks the BVH with the t interval widened by a slack that keeps boxes whose
 * face holds the hit point, so it is meant for statistics on large scenes. */
void rb2o_tie_count_brute(const uint32_t* woop, const uint32_t* triidx, uint32_t n_woop_u4, const float* rays,
                          uint32_t n, const rb2o_hit* hits, uint32_t* out, int nthreads);
void rb2o_tie_count(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx, const float* rays,
                    uint32_t n, const rb2o_hit* hits, uint32_t* out, int nthreads);

/* The synthetic heightfield workload (oracle copy of the product generator;
 * rb2_oracle_gen.c).  Return 0 on success. */
int rb2o_gen_heightfield_counts(uint32_t grid_n, uint32_t n_boxes, uint32_t* nv, uint32_t* ntri);
int rb2o_gen_heightfield(uint64_t seed, uint32_t grid_n, float amplitude, uint32_t n_boxes, float box_min,
                         float box_max, float* v, uint32_t* idx);
int rb2o_gen_surface_rays(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, uint64_t seed,
                          uint64_t n_rays, float offset_scale, float anyhit_fraction, float* rays, uint8_t* flags);

/* Intersection record of a closest hit, as the reference's bulk kernel fills
 * IntersectionBuffer (accelerators/sbvh/kepler_dynamic_fetch.h:313-355),
 * in IEEE single precision with no contraction:
 *   Ng  = normalize(cross(v1 - v0, v2 - v0)), normalize(x) = x * (1/sqrtf(dot(x,x)))
 *         (core/primitives.h:267-270), dot = (x.x*y.x + x.y*y.y) + x.z*y.z
 *   Ns  = Ng (the generated scenes carry no vertex normals)
 *   position = o + d * t;  wi = -d;  front = dot(Ng, d) < 0
 *   uv = (u, v) of the accepted triangle;  epsilon = 1e-3f * t
 *   intersected = 1 on a hit, 0 on a miss or a masked ray; other fields are
 *   left untouched on a miss.
 * tris: 4 words per triangle (3 vertex indices, material id). */
typedef struct {
    float* position;      /* 3 per ray (SoA planes: x[n], y[n], z[n]) */
    float* ng;
    float* ns;
    float* wi;
    float* uv;            /* 2 per ray, interleaved */
    uint32_t* prim;
    uint32_t* material;
    uint8_t* front;
    uint8_t* intersected;
    float* epsilon;
} rb2o_isect_soa;
void rb2o_isect(const float* verts, const uint32_t* tris4, const float* rays, const rb2o_hit* hits, uint32_t n,
                rb2o_isect_soa* out);

/* Film reconstruction (renderers/samplerrenderer.cu:103-168, core/film.cpp:36-93,
 * core/filter.h:46-132) with the table indexed by x and y, in IEEE single
 * precision with no contraction:
 *   table[y][x] = filter(((x + 0.5) * xw) / 16, ((y + 0.5) * yw) / 16)
 *     box 1; triangle max(0, xw - |x|) max(0, yw - |y|);
 *     Gaussian max(0, exp(-a x x) - exp(-a xw xw)) * (same in y)
 *   sample s (raster position) reaches pixel (px, py) when
 *     ceil(s.x - 0.5 - xw) <= px <= floor(s.x - 0.5 + xw) (and in y);
 *   w = table[min(floor(|(py - (s.y - 0.5)) * (1/yw) * 16|), 15)]
 *              [min(floor(|(px - (s.x - 0.5)) * (1/xw) * 16|), 15)]
 *   pixel = max(0, sum(w L) * (1 / sum(w))), 0 when sum(w) = 0; the sums run
 *   over neighbour rows, then columns, then samples, in increasing order.
 * kind 0 = mean of the pixel's own samples (sum * (1/spp)).
 * Samples are sample-major: sample j of pixel p at j * w * h + p. */
void rb2o_filter_table(uint32_t kind, float xw, float yw, float alpha, float* table256);
void rb2o_film(uint32_t kind, float xw, float yw, float alpha, uint32_t width, uint32_t height, uint32_t spp,
               const float* xy, const float* L4, float* rgb);

/* ---- shading references (FP64 accumulation) ---------------------------------
 * Scene for the integrator references: vertices (xyz), triangles (3 indices),
 * per-triangle material, per-material albedo/emission (rgb), emissive
 * triangle list (uniform light choice, integrators/integrator_path.cu:122). */
/* A layered material in the product's rb2_material_desc layout: bxdf layers
 * (0 Lambertian, 1 Oren-Nayar, 2 mirror, 3 glass, 4 Blinn microfacet; Fresnel
 * 0 dielectric, 1 conductor, 2 none) following core/reflection.cu:42-299 and
 * core/material.cu:56-326, with the two documented differences of the
 * product: a sampled multi-layer pdf is divided by the layer count, and a
 * glass layer adds no microfacet term. */
typedef struct {
    uint32_t type, fresnel;
    float color[3], sigma_deg, etai, etat, exponent, eta[3], k[3];
} rb2o_layer;
typedef struct {
    uint32_t n_layers, reserved;
    rb2o_layer layer[4];
} rb2o_material;

typedef struct {
    const float* verts;
    const uint32_t* tris;
    const uint32_t* tri_mat;
    const float* albedo;
    const float* emission;
    const uint32_t* lights;
    uint32_t n_lights;
    const rb2o_material* materials;  /* nullable: one Lambertian layer (albedo) per material */
} rb2o_scene;

/* The material functions in FP64 on world-space directions around normal n:
 * sample == 0: q = (n, wo, wi) -> out = (f rgb, pdf), specular layers excluded;
 * sample != 0: q = (n, wo, u1, u2, uc) -> out = (wi, f rgb, pdf, specular). */
void rb2o_material_query(const rb2o_material* m, int sample, const double* q, double* out);

typedef struct {
    const uint32_t* nodes;
    const uint32_t* woop;
    const uint32_t* triidx;
} rb2o_bvh;

/* Visit counters of the integrator references (ao, pt, bdpt) per ray type:
 * out[type * 4 + k], k = nodes, triangles, leaf terminators, rays.  Counting
 * is off until rb2o_counts_reset(1). */
enum { RB2O_RAY_CAMERA = 0, RB2O_RAY_EXTENSION = 1, RB2O_RAY_SHADOW = 2, RB2O_RAY_CONNECTION = 3, RB2O_RAY_LIGHT = 4,
       RB2O_RAY_TYPES = 5 };
void rb2o_counts_reset(int on);
void rb2o_counts_read(uint64_t* out);

/* Ambient occlusion (integrators/integrator_ao.cu:51-84): per primary ray, the
 * unoccluded fraction of `samples` cosine-distributed rays about the
 * viewer-facing geometric normal, tmin 1e-3 t, tmax radius; 0 on a miss.
 * compat bit 1: the reference's direction formula about the unflipped normal
 * (core/montecarlo.cu:133-151; a sample whose X axis is undefined is open). */
void rb2o_ao(const rb2o_bvh* b, const rb2o_scene* s, const float* prim_rays, uint32_t n, uint32_t samples,
             float radius, uint64_t seed, uint32_t compat, double* out, int nthreads);
/* The two reference formulas the compatibility modes restate, in double (pinned
 * against the reference's compiled functions by the CPU tests):
 * rb2o_ao_ref_dir: the AO direction about n3 (0 where the reference's is NaN);
 * rb2o_light_le_ref: DiffuseAreaLight::Le's direction and Le / pdf factor. */
int rb2o_ao_ref_dir(const double* n3, double u1, double u2, double* out3);
void rb2o_light_le_ref(const double* ln3, double area, double u3, double u4, double* dir3, double* k);

/* One path-traced sample per camera ray (integrators/integrator_path.cu:56-260
 * with unbiased Russian roulette): NEE to a uniformly chosen emissive triangle
 * and BSDF sampling combined by the balance heuristic; out_rgb: 3 per ray.
 * compat bit 2: roulette from bounce rr_start + 1 dividing survivors by 1 - q
 * (integrator_path.cu:232-244); bit 4: the same NEE draws at every vertex
 * (integrator_path.cu:113). */
void rb2o_pt(const rb2o_bvh* b, const rb2o_scene* s, const float* rays, uint32_t n, uint32_t max_depth,
             uint32_t rr_start, float rr_prob, uint64_t seed, uint32_t compat, double* out_rgb, int nthreads);

/* BDPT with a light-vertex cache (integrators/integrator_bdpt_lvc_sk.cu:47-514,
 * with uniform 1/k weights over all k strategies of a k-segment path and the
 * cache-size factor): n_iter iterations, each tracing n_light_paths light
 * subpaths into the cache and one camera path per camera ray
 * (cam_rays: n_iter x n_cam rays, iteration-major).  out_rgb: mean over
 * iterations, 3 per camera pixel. */
void rb2o_bdpt(const rb2o_bvh* b, const rb2o_scene* s, const float* cam_rays, uint32_t n_cam, uint32_t n_iter,
               uint32_t n_light_paths, uint32_t K, uint32_t C, uint32_t rr_start, float rr_prob, uint64_t seed,
               double* out_rgb, int nthreads);

/* The reference's own BDPT estimator (integrators/integrator_bdpt_lvc_sk.cu:47-514),
 * restated in FP64 with counter-keyed draws: a preparation pass of n_prep
 * light subpaths sizes the cache at ceil(1.1 * mean stored vertices *
 * n_light_paths) (single precision, :466-470; n_prep 0: no cap); light
 * subpaths start as DiffuseAreaLight::Le (core/lights.cu:63-69: direction
 * uniform about world +z, negated, contribution Le / pdf without the triangle
 * choice), store every surface vertex (emitters with zero contribution, then
 * stop), play roulette min(1, luminance) at every bounce and stop when black,
 * keeping at most light_max_depth vertices; camera vertices 0..cam_max_depth
 * add emission (first vertex or after a specular bounce), NEE at full weight
 * with the first vertex's draws at every vertex, and `connections`
 * connections to uniform cached vertices weighted 1 / ((bounce + 1) + depth);
 * camera roulette from bounce cam_rrstart + 1 divides survivors by 1 - q. */
typedef struct {
    uint32_t n_prep, n_light_paths, light_max_depth, cam_max_depth, cam_rrstart, connections;
    float cam_rrprob;
} rb2o_bdpt_ref_params;
void rb2o_bdpt_ref(const rb2o_bvh* b, const rb2o_scene* s, const float* cam_rays, uint32_t n_cam, uint32_t n_iter,
                   const rb2o_bdpt_ref_params* p, uint64_t seed, double* out_rgb, int nthreads);

/* PCG32 (O'Neill 2014, pcg32_srandom_r / pcg32_random_r), the generator the
 * product uses for every seeded stream. */
typedef struct { uint64_t state, inc; } rb2o_pcg32;
void rb2o_pcg32_seed(rb2o_pcg32* r, uint64_t initstate, uint64_t initseq);
uint32_t rb2o_pcg32_next(rb2o_pcg32* r);

#ifdef __cplusplus
}
#endif
#endif
