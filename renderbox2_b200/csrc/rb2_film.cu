// Film: filtered, deterministic image reconstruction (rb2_film_develop, the
// integrators' filtered accumulation) and the PFM image writer.
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_film.cuh"
#include "rb2_internal.h"
#include "rb2_render.h"
#include "rb2_render_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace rb2dev {

// The integrators' default (RB2_FILTER_NONE): mean of the pixel's own samples.
__global__ void k_film_mean(const float4* L, uint32_t npix, uint32_t spp, float* rgb)
{
    const float inv = 1.0f / (float)spp;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (uint32_t j = 0; j < spp; j++) {
            const float4 l = L[(size_t)j * npix + pix];
            ax = __fadd_rn(ax, l.x);
            ay = __fadd_rn(ay, l.y);
            az = __fadd_rn(az, l.z);
        }
        rgb[3 * (size_t)pix + 0] = __fmul_rn(ax, inv);
        rgb[3 * (size_t)pix + 1] = __fmul_rn(ay, inv);
        rgb[3 * (size_t)pix + 2] = __fmul_rn(az, inv);
    }
}

}  // namespace rb2dev

using namespace rb2;

namespace {

int cuda_fail(cudaError_t e, const char* what) { return fail(rb2::cuda_status(e), std::string(what) + ": " + cudaGetErrorString(e)); }

unsigned film_grid(uint64_t npix)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((npix + 255) / 256, (uint64_t)sms * 8));
}

}  // namespace

namespace rb2 {

int film_args(const rb2_filter& f, uint32_t width, uint32_t height, rb2dev::FilmArgs& out)
{
    int rc = rb2_filter_table(&f, out.table);
    if (rc) return rc;
    out.xw = f.xwidth;
    out.yw = f.ywidth;
    out.inv_xw = 1.0f / f.xwidth;
    out.inv_yw = 1.0f / f.ywidth;
    // A sample of pixel q lies within 0.5 + width of q's centre row/column;
    // one more pixel covers rounding of s - 0.5 -/+ width.
    out.rx = (int)std::floor(f.xwidth + 0.5f) + 1;
    out.ry = (int)std::floor(f.ywidth + 0.5f) + 1;
    out.width = width;
    out.height = height;
    return RB2_OK;
}

}  // namespace rb2

extern "C" {

int rb2_film_develop(const rb2_filter* f, uint32_t width, uint32_t height, uint32_t spp, const float* d_xy,
                     const float* d_L, float* d_rgb, void* stream)
{
    int rc = validate_filter(f);
    if (rc) return rc;
    const uint64_t npix = (uint64_t)width * height;
    if (npix == 0 || spp == 0) return RB2_OK;
    if (npix * spp > 0xFFFFFFFFull) return fail(RB2_EINVAL, "width x height x spp must be < 2^32");
    if (!d_L || !d_rgb || (f->kind != RB2_FILTER_NONE && !d_xy)) return fail(RB2_EINVAL, "null buffer");
    if (((uintptr_t)d_L & 15u) || ((uintptr_t)d_xy & 7u)) return fail(RB2_EINVAL, "L must be 16-byte and xy 8-byte aligned");
    const cudaStream_t s = (cudaStream_t)stream;
    const unsigned g = film_grid(npix);
    if (f->kind == RB2_FILTER_NONE) {
        rb2dev::k_film_mean<<<g, 256, 0, s>>>(reinterpret_cast<const float4*>(d_L), (uint32_t)npix, spp, d_rgb);
    } else {
        rb2dev::FilmArgs fa{};
        if ((rc = film_args(*f, width, height, fa))) return rc;
        rb2dev::k_film_gather<<<g, 256, 0, s>>>(fa, rb2dev::ArrayPos{reinterpret_cast<const float2*>(d_xy), (uint32_t)npix},
                                                reinterpret_cast<const float4*>(d_L), spp, nullptr, d_rgb);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RB2_OK : cuda_fail(e, "film launch");
}

int rb2_integrator_set_filter(rb2_integrator* it, const rb2_filter* f)
{
    if (!it) return fail(RB2_EINVAL, "null integrator");
    if (!f) {
        it->filter = rb2_filter{RB2_FILTER_NONE, 0.5f, 0.5f, 0.0f};
        return RB2_OK;
    }
    const int rc = validate_filter(f);
    if (rc) return rc;
    it->filter = *f;
    return RB2_OK;
}

int rb2_image_write_pfm(const char* path, const float* h_rgb, uint32_t width, uint32_t height)
{
    if (!path || (!h_rgb && width && height)) return fail(RB2_EINVAL, "null argument");
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(RB2_EIO, std::string("cannot open ") + path);
    // PFM: "PF", dimensions, negative scale = little-endian, rows bottom to top.
    const int ok_header = std::fprintf(fp, "PF\n%u %u\n-1.0\n", width, height) > 0;
    bool ok = ok_header;
    for (uint32_t row = 0; ok && row < height; row++) {
        const float* src = h_rgb + 3 * (size_t)(height - 1 - row) * width;
        ok = std::fwrite(src, sizeof(float), 3 * (size_t)width, fp) == 3 * (size_t)width;
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? RB2_OK : fail(RB2_EIO, std::string("write failed: ") + path);
}

}  // extern "C"
