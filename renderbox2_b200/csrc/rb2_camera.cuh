// Camera-ray generation shared by the tracer and the integrators.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rb2dev {

struct CamArgs {
    float r2c[16];
    float c2w[16];
    uint32_t width, height, spp, jitter;
    uint64_t seed;
};

// Row-vector products evaluated left to right without contraction, like the
// reference's float4 dot (helper_math) on Matrix4x4 rows (core/transform.h:186-199).
__device__ __forceinline__ float row_dot(const float* r, float x, float y, float z, float w)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r[0], x), __fmul_rn(r[1], y)), __fmul_rn(r[2], z)), __fmul_rn(r[3], w));
}

__device__ __forceinline__ void camera_ray(const float* r2c, const float* c2w, float x, float y, float4& o4, float4& d4)
{
    // p_camera = raster_to_camera(point (x, y, 0)), divided by w (core/camera.cu:91-98).
    float px = row_dot(r2c + 0, x, y, 0.0f, 1.0f);
    float py = row_dot(r2c + 4, x, y, 0.0f, 1.0f);
    float pz = row_dot(r2c + 8, x, y, 0.0f, 1.0f);
    float pw = row_dot(r2c + 12, x, y, 0.0f, 1.0f);
    px = __fdiv_rn(px, pw); py = __fdiv_rn(py, pw); pz = __fdiv_rn(pz, pw);
    // normalize = v * (1 / sqrt(dot(v, v)))
    float dd = __fadd_rn(__fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py)), __fmul_rn(pz, pz));
    float inv = __fdiv_rn(1.0f, __fsqrt_rn(dd));
    float dxc = __fmul_rn(px, inv), dyc = __fmul_rn(py, inv), dzc = __fmul_rn(pz, inv);
    // camera_to_world: origin as a point, direction as a vector.
    float oxw = row_dot(c2w + 0, 0.0f, 0.0f, 0.0f, 1.0f);
    float oyw = row_dot(c2w + 4, 0.0f, 0.0f, 0.0f, 1.0f);
    float ozw = row_dot(c2w + 8, 0.0f, 0.0f, 0.0f, 1.0f);
    float oww = row_dot(c2w + 12, 0.0f, 0.0f, 0.0f, 1.0f);
    o4 = make_float4(__fdiv_rn(oxw, oww), __fdiv_rn(oyw, oww), __fdiv_rn(ozw, oww), 0.0f);
    d4 = make_float4(row_dot(c2w + 0, dxc, dyc, dzc, 0.0f), row_dot(c2w + 4, dxc, dyc, dzc, 0.0f),
                     row_dot(c2w + 8, dxc, dyc, dzc, 0.0f), 3.402823466e+38f);
}

__device__ __forceinline__ uint32_t pcg_hash(uint64_t v)
{
    // One PCG32 output step applied to a counter (O'Neill 2014 output function).
    uint64_t state = v * 6364136223846793005ULL + 1442695040888963407ULL;
    uint32_t xs = (uint32_t)(((state >> 18u) ^ state) >> 27u);
    uint32_t rot = (uint32_t)(state >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}

}  // namespace rb2dev
