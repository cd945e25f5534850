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

#ifdef __cplusplus
}
#endif
#endif
