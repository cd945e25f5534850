// Film reconstruction on the device: every output pixel gathers the samples
// of its neighbourhood in a fixed order (rows, columns, then samples), so the
// image does not depend on scheduling.  The weights follow the reference's
// splat (renderers/samplerrenderer.cu:103-168): a sample with raster position
// s contributes to pixel x when ceil(s - 0.5 - width) <= x <= floor(s - 0.5 +
// width), with weight table[min(floor(|x - (s - 0.5)| / width * 16), 15)].
// Arithmetic is IEEE single precision with no contraction (the oracle's
// rb2o_film restates it operation by operation).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb2_shading.cuh"

namespace rb2dev {

struct FilmArgs {
    float table[256];
    float xw, yw, inv_xw, inv_yw;
    int rx, ry;                 // neighbourhood half-size in pixels
    uint32_t width, height;
};

// Sample positions from a buffer, sample-major (sample j of pixel p at j * npix + p).
struct ArrayPos {
    const float2* xy;
    uint32_t npix;
    __device__ __forceinline__ float2 operator()(uint32_t j, uint32_t pix) const { return xy[(size_t)j * npix + pix]; }
};

// accum == nullptr: write max(0, sum(wL) / sum(w)) to rgb; otherwise add the
// sums to accum (rgb, weight) in fixed order.
template <class Pos>
__global__ void k_film_gather(const __grid_constant__ FilmArgs f, Pos pos, const float4* L, uint32_t per_pixel,
                              float4* accum, float* rgb)
{
    __shared__ float tab[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) tab[i] = f.table[i];
    __syncthreads();
    const uint32_t W = f.width, H = f.height, npix = W * H;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        const int x = (int)(pix % W), y = (int)(pix / W);
        const float xf = (float)x, yf = (float)y;
        float ax = 0.0f, ay = 0.0f, az = 0.0f, aw = 0.0f;
        const int qy0 = max(0, y - f.ry), qy1 = min((int)H - 1, y + f.ry);
        const int qx0 = max(0, x - f.rx), qx1 = min((int)W - 1, x + f.rx);
        for (int qy = qy0; qy <= qy1; qy++) {
            for (int qx = qx0; qx <= qx1; qx++) {
                const uint32_t q = (uint32_t)qy * W + (uint32_t)qx;
                for (uint32_t j = 0; j < per_pixel; j++) {
                    const float2 s = pos(j, q);
                    const float dx = __fsub_rn(s.x, 0.5f), dy = __fsub_rn(s.y, 0.5f);
                    if (x < (int)ceilf(__fsub_rn(dx, f.xw)) || x > (int)floorf(__fadd_rn(dx, f.xw)) ||
                        y < (int)ceilf(__fsub_rn(dy, f.yw)) || y > (int)floorf(__fadd_rn(dy, f.yw)))
                        continue;
                    const float fx = fabsf(__fmul_rn(__fmul_rn(__fsub_rn(xf, dx), f.inv_xw), 16.0f));
                    const float fy = fabsf(__fmul_rn(__fmul_rn(__fsub_rn(yf, dy), f.inv_yw), 16.0f));
                    const int ix = min((int)floorf(fx), 15), iy = min((int)floorf(fy), 15);
                    const float w = tab[iy * 16 + ix];
                    const float4 l = L[(size_t)j * npix + q];
                    ax = __fadd_rn(ax, __fmul_rn(w, l.x));
                    ay = __fadd_rn(ay, __fmul_rn(w, l.y));
                    az = __fadd_rn(az, __fmul_rn(w, l.z));
                    aw = __fadd_rn(aw, w);
                }
            }
        }
        if (accum) {
            const float4 a = accum[pix];
            accum[pix] = make_float4(__fadd_rn(a.x, ax), __fadd_rn(a.y, ay), __fadd_rn(a.z, az), __fadd_rn(a.w, aw));
        } else {
            const float inv = aw != 0.0f ? __fdiv_rn(1.0f, aw) : 0.0f;
            rgb[3 * (size_t)pix + 0] = fmaxf(0.0f, __fmul_rn(ax, inv));
            rgb[3 * (size_t)pix + 1] = fmaxf(0.0f, __fmul_rn(ay, inv));
            rgb[3 * (size_t)pix + 2] = fmaxf(0.0f, __fmul_rn(az, inv));
        }
    }
}

// Final image of an accumulated film.
static __global__ void k_film_resolve(const float4* accum, uint32_t npix, float* rgb)
{
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        const float4 a = accum[pix];
        const float inv = a.w != 0.0f ? __fdiv_rn(1.0f, a.w) : 0.0f;
        rgb[3 * (size_t)pix + 0] = fmaxf(0.0f, __fmul_rn(a.x, inv));
        rgb[3 * (size_t)pix + 1] = fmaxf(0.0f, __fmul_rn(a.y, inv));
        rgb[3 * (size_t)pix + 2] = fmaxf(0.0f, __fmul_rn(a.z, inv));
    }
}

}  // namespace rb2dev
