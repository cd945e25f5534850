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

#include "rb2_render.h"

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

/* ----------------------------------------------------------- scene files --
 * Loads the reference's scene description: the XML schema of
 * io/customfilereader.cpp:47-291 (<scene> with <files><count>1</count>
 * <file>x.obj</file></files>, <material><name/><bsdf><layers/><bxdf><type/>
 * <reflectance/>...</bxdf></bsdf></material>..., <object><name/><material/>
 * </object>..., <lightobjects><light><name/><type/><Le/></light>...
 * </lightobjects>, <camera><position/><lookat/><up/><fov/></camera>), or a
 * bare Wavefront OBJ (io/objfilereader.cpp).  Mesh = OBJ object ("o name");
 * indices are file-global, as the reference keeps them.  Materials keep the
 * reference's numbering: XML materials in order, then one emitter material
 * per light.  Triangle material = its object's material, the light's
 * emitter material for light meshes, 0 for meshes the file does not name.
 * Differences: a face of n > 3 vertices is fan-triangulated (the reference
 * kept its first triangle), negative (relative) OBJ indices are accepted,
 * '#' starts a comment anywhere on a line (the reference skipped any line
 * containing '#'), geometry before the first "o" goes to a mesh named
 * "default", and <fov> is read when present (the reference used 90).  Every
 * material's layers (up to 4 bxdf entries, MAX_LAYERS in core/material.h)
 * are returned as rb2_material_desc for rb2_scene_set_materials; emitter
 * materials have no layers. */
typedef struct rb2_scene_file rb2_scene_file;
typedef struct {
    uint32_t n_vertices, n_triangles, n_materials, n_lights, n_meshes;
    int32_t has_camera;
    float eye[3], lookat[3], up[3];
    float fov_deg;
} rb2_scene_file_info;
int rb2_scene_file_load(const char* path, rb2_scene_file** out);  /* .xml or .obj */
int rb2_scene_file_info_get(const rb2_scene_file* f, rb2_scene_file_info* out);
const float* rb2_scene_file_vertices(const rb2_scene_file* f);        /* 3 floats per vertex */
const uint32_t* rb2_scene_file_indices(const rb2_scene_file* f);      /* 3 per triangle */
const uint32_t* rb2_scene_file_tri_material(const rb2_scene_file* f); /* 1 per triangle */
const float* rb2_scene_file_albedo(const rb2_scene_file* f);          /* 3 per material */
const float* rb2_scene_file_emission(const rb2_scene_file* f);        /* 3 per material */
const uint32_t* rb2_scene_file_bsdf_types(const rb2_scene_file* f);   /* first layer's RB2_BSDF_* per material */
const rb2_material_desc* rb2_scene_file_materials(const rb2_scene_file* f);  /* one per material */
/* Mesh i: name and its triangle range [first, first + count). */
int rb2_scene_file_mesh(const rb2_scene_file* f, uint32_t i, const char** name, uint32_t* first, uint32_t* count);
void rb2_scene_file_free(rb2_scene_file* f);

/* PCG32 stream (O'Neill 2014): 32-bit outputs, for tests of seeding. */
int rb2_pcg32_fill(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif
#endif
