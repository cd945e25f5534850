/*
 * rb2_scene.h -- seeded synthetic scenes and ray sets (host side).
 *
 * The reference ships no scenes; its loaders (io/customfilereader.cpp,
 * io/objfilereader.cpp) read XML/OBJ files that are absent.  These generators
 * make the workloads with fixed seeds (PCG32, O'Neill 2014) so the CPU
 * oracle and the device kernels see identical inputs.
 */
#ifndef RB2_SCENE_H
#define RB2_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Heightfield over the unit square (grid_n x grid_n cells, two triangles per
 * cell, up-facing), y = amplitude * fractal value noise, plus n_boxes
 * axis-aligned boxes (12 triangles each, outward facing) with edge lengths
 * uniform in [box_min, box_max] resting on or just above the field.
 * Sizes: nv = (grid_n+1)^2 + 8*n_boxes, ntri = 2*grid_n^2 + 12*n_boxes. */
int rb2_gen_heightfield_counts(uint32_t grid_n, uint32_t n_boxes, uint32_t* nv, uint32_t* ntri);
int rb2_gen_heightfield(uint64_t seed, uint32_t grid_n, float amplitude, uint32_t n_boxes, float box_min,
                        float box_max, float* v_xyz, uint32_t* idx3);

/* Closed room [0,1]^3 (inward-facing walls) with n_boxes boxes and
 * n_spheres icospheres (subdivision `sphere_subdiv`, 20*4^s triangles each,
 * radii log-uniform in [rmin, rmax]) and n_lights quad area lights (2
 * triangles each) just below the ceiling.  Material id per triangle:
 * 0..n_albedo-1 diffuse, the last n_lights ids are emitters (one per light).
 * Sizes from rb2_gen_room_counts. */
int rb2_gen_room_counts(uint32_t n_boxes, uint32_t n_spheres, uint32_t sphere_subdiv, uint32_t n_lights,
                        uint32_t* nv, uint32_t* ntri);
int rb2_gen_room(uint64_t seed, uint32_t n_boxes, uint32_t n_spheres, uint32_t sphere_subdiv, float rmin,
                 float rmax, uint32_t n_lights, float* v_xyz, uint32_t* idx3, uint32_t* tri_material);

/* Incoherent "diffuse bounce" rays: origins uniform by area on the surface,
 * offset along the geometric normal by offset_scale * scene diagonal,
 * directions cosine-distributed about that normal, tmin 0, tmax FLT_MAX.
 * rays: 8 floats per ray.  flags (nullable): 1 = any-hit ray, 0 = closest-hit,
 * drawn with probability anyhit_fraction.  Multi-threaded. */
int rb2_gen_surface_rays(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, uint64_t seed,
                         uint64_t n_rays, float offset_scale, float anyhit_fraction, float* rays, uint8_t* flags);

/* PCG32 stream (O'Neill 2014): 32-bit outputs, for tests of seeding. */
int rb2_pcg32_fill(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif
#endif
