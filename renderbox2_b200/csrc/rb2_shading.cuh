// Device shading helpers: counter-based random numbers, frames and the
// sampling routines of the reference's core/montecarlo.cu and
// core/reflection.cu restated for the integrators.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rb2dev {

// ---- random numbers -----------------------------------------------------------------
// Counter-based: every draw is a pure function of (seed, stream key, dimension),
// so results do not depend on which warp or launch traced a path.  Mixing is
// splitmix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) followed by the PCG32 output permutation
// (O'Neill 2014).
__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ float rng_u01(uint64_t seed, uint64_t key, uint32_t dim)
{
    const uint64_t s = splitmix64(seed ^ splitmix64(key * 0x100000001B3ull + dim));
    const uint32_t xs = (uint32_t)(((s >> 18u) ^ s) >> 27u);
    const uint32_t rot = (uint32_t)(s >> 59u);
    const uint32_t r = (xs >> rot) | (xs << ((0u - rot) & 31u));
    return (float)(r >> 8) * (1.0f / 16777216.0f);  // [0, 1)
}

// ---- vectors ----------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mul3(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 v) { return mul(v, rsqrtf(dot3(v, v))); }
__device__ __forceinline__ float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }

// Frame::set_from_z (core/primitives.h:231-237): X, Y, Z with Z = n.
struct Frame {
    float3 x, y, z;
};
__device__ __forceinline__ Frame frame_from_z(float3 n)
{
    Frame f;
    f.z = normalize3(n);
    const float3 t = fabsf(f.z.x) > 0.99f ? f3(0, 1, 0) : f3(1, 0, 0);
    f.y = normalize3(cross3(f.z, t));
    f.x = cross3(f.y, f.z);
    return f;
}
__device__ __forceinline__ float3 to_world(const Frame& f, float3 w)
{
    return add(add(mul(f.x, w.x), mul(f.y, w.y)), mul(f.z, w.z));
}

// concentric_sample_disk (core/montecarlo.cu:59-106, Shirley & Chiu 1997).
__device__ __forceinline__ float2 concentric_disk(float u1, float u2)
{
    const float sx = 1.0f - 2.0f * u1, sy = 1.0f - 2.0f * u2;
    if (sx == 0.0f && sy == 0.0f) return make_float2(0.0f, 0.0f);
    float r, theta;
    if (sx >= -sy) {
        if (sx > sy) { r = sx; theta = sy > 0.0f ? sy / r : 8.0f + sy / r; }
        else { r = sy; theta = 2.0f - sx / r; }
    } else {
        if (sx <= sy) { r = -sx; theta = 4.0f - sy / r; }
        else { r = -sy; theta = 6.0f + sx / r; }
    }
    theta *= 0.78539816339744831f;  // pi / 4
    float s, c;
    __sincosf(theta, &s, &c);
    return make_float2(r * c, r * s);
}

// cosine_sample_hemisphere (core/montecarlo.cu:153-158): local z-up direction.
__device__ __forceinline__ float3 cosine_hemisphere(float u1, float u2)
{
    const float2 d = concentric_disk(u1, u2);
    return f3(d.x, d.y, sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y)));
}

// uniform_sample_triangle (core/montecarlo.cu:165-172): barycentrics (b0, b1).
__device__ __forceinline__ float3 sample_triangle(float3 v0, float3 v1, float3 v2, float u1, float u2)
{
    const float su = sqrtf(u1);
    const float b0 = 1.0f - su, b1 = u2 * su;
    return add(add(mul(v0, b0), mul(v1, b1)), mul(v2, 1.0f - b0 - b1));
}

__device__ __forceinline__ float luminance(float3 c)
{
    // core/util.h:161-169
    return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z;
}

constexpr float kInvPi = 0.31830988618379067154f;

}  // namespace rb2dev
