// Stand-in for the CUDA Samples "helper_math.h" header that the reference
// includes (core/primitives.h:27) but does not ship.  Written from the plain
// definitions of 2/3/4-component vector arithmetic; used only to compile the
// reference's host SBVH builder and Compact2 packer in place as a test oracle.
//
// Arithmetic contract (the product's packer uses the same definitions, so the
// Woop coefficients of both are bit-identical):
//   dot(a,b)    = a.x*b.x + a.y*b.y + a.z*b.z            (left to right, no FMA)
//   cross(a,b)  = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   normalize(v)= v * (1.0f / sqrtf(dot(v,v)))
//   lerp(a,b,t) = a + t*(b-a)
//   clamp(f,a,b)= fmaxf(a, fminf(f,b))
#ifndef RB2_ORACLE_HELPER_MATH_H
#define RB2_ORACLE_HELPER_MATH_H

#include <cuda_runtime.h>
#include <vector_types.h>
#include <vector_functions.h>
#include <cmath>
#include <algorithm>

typedef unsigned int uint;

#ifndef __CUDACC__
inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
#endif

// ---- scalar helpers ---------------------------------------------------------
inline float lerp(float a, float b, float t) { return a + t * (b - a); }
inline float clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
inline int clamp(int f, int a, int b) { return std::max(a, std::min(f, b)); }

// ---- constructors -------------------------------------------------------------
inline float2 make_float2(float s) { return make_float2(s, s); }
inline float3 make_float3(float s) { return make_float3(s, s, s); }
inline float3 make_float3(const float4& a) { return make_float3(a.x, a.y, a.z); }
inline float3 make_float3(const float2& a, float z) { return make_float3(a.x, a.y, z); }
inline float3 make_float3(const int3& a) { return make_float3(float(a.x), float(a.y), float(a.z)); }
inline float4 make_float4(float s) { return make_float4(s, s, s, s); }
inline float4 make_float4(const float3& a, float w) { return make_float4(a.x, a.y, a.z, w); }
inline float4 make_float4(const float3& a) { return make_float4(a.x, a.y, a.z, 0.0f); }
inline int3 make_int3(int s) { return make_int3(s, s, s); }
inline uint3 make_uint3(uint s) { return make_uint3(s, s, s); }
inline uint4 make_uint4(uint s) { return make_uint4(s, s, s, s); }

// ---- float2 -------------------------------------------------------------------
inline float2 operator+(const float2& a, const float2& b) { return make_float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(const float2& a, const float2& b) { return make_float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(const float2& a, float s) { return make_float2(a.x * s, a.y * s); }
inline float2 operator*(float s, const float2& a) { return make_float2(a.x * s, a.y * s); }

// ---- float3 -------------------------------------------------------------------
inline float3 operator-(const float3& a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator+(const float3& a, const float3& b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator+(const float3& a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
inline float3 operator-(const float3& a, const float3& b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator-(const float3& a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
inline float3 operator*(const float3& a, const float3& b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator*(const float3& a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, const float3& a) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(const float3& a, const float3& b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator/(const float3& a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator/(float s, const float3& a) { return make_float3(s / a.x, s / a.y, s / a.z); }
inline void operator+=(float3& a, const float3& b) { a.x += b.x; a.y += b.y; a.z += b.z; }
inline void operator-=(float3& a, const float3& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
inline void operator*=(float3& a, float s) { a.x *= s; a.y *= s; a.z *= s; }
inline void operator*=(float3& a, const float3& b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; }
inline void operator/=(float3& a, float s) { a.x /= s; a.y /= s; a.z /= s; }

inline float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(const float3& a, const float3& b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(const float3& v) { return sqrtf(dot(v, v)); }
inline float3 normalize(const float3& v) { float inv_len = rsqrtf(dot(v, v)); return v * inv_len; }
inline float3 fminf(const float3& a, const float3& b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
inline float3 fmaxf(const float3& a, const float3& b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
inline float3 lerp(const float3& a, const float3& b, float t) { return a + t * (b - a); }
inline float3 clamp(const float3& v, float a, float b) { return make_float3(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b)); }
inline float3 fabs(const float3& v) { return make_float3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }

// ---- float4 -------------------------------------------------------------------
inline float4 operator-(const float4& a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
inline float4 operator+(const float4& a, const float4& b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator-(const float4& a, const float4& b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline float4 operator*(const float4& a, const float4& b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline float4 operator*(const float4& a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator*(float s, const float4& a) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator/(const float4& a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
inline void operator+=(float4& a, const float4& b) { a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w; }
inline void operator*=(float4& a, const float4& b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; a.w *= b.w; }
inline void operator*=(float4& a, float s) { a.x *= s; a.y *= s; a.z *= s; a.w *= s; }
inline void operator/=(float4& a, float s) { a.x /= s; a.y /= s; a.z /= s; a.w /= s; }
inline float dot(const float4& a, const float4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// ---- int3 ---------------------------------------------------------------------
inline int3 clamp(const int3& v, int a, int b) { return make_int3(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b)); }
inline int3 clamp(const int3& v, const int3& a, const int3& b)
{
    return make_int3(clamp(v.x, a.x, b.x), clamp(v.y, a.y, b.y), clamp(v.z, a.z, b.z));
}

#endif
