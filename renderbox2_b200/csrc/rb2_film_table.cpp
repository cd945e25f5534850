// Filter table of the film (core/film.cpp:36-60 with core/filter.h:46-132),
// computed on the host in IEEE single precision without contraction.  The
// table is indexed [y][x] with fx taken from x (the reference took it from y,
// core/film.cpp:56, so its table did not vary along x).
#include "rb2_internal.h"
#include "rb2_render.h"

#include <cmath>

namespace {

float eval_filter(const rb2_filter& f, float x, float y)
{
    switch (f.kind) {
    case RB2_FILTER_TRIANGLE:
        return std::fmax(0.0f, f.xwidth - std::fabs(x)) * std::fmax(0.0f, f.ywidth - std::fabs(y));
    case RB2_FILTER_GAUSSIAN: {
        const float expx = std::exp(-f.alpha * f.xwidth * f.xwidth);
        const float expy = std::exp(-f.alpha * f.ywidth * f.ywidth);
        const float gx = std::fmax(0.0f, std::exp(-f.alpha * x * x) - expx);
        const float gy = std::fmax(0.0f, std::exp(-f.alpha * y * y) - expy);
        return gx * gy;
    }
    default:
        return 1.0f;  // box (and "none", unused)
    }
}

}  // namespace

namespace rb2 {

int validate_filter(const rb2_filter* f)
{
    if (!f) return fail(RB2_EINVAL, "null filter");
    if (f->kind > RB2_FILTER_GAUSSIAN) return fail(RB2_EINVAL, "unknown filter kind");
    if (f->kind == RB2_FILTER_NONE) return RB2_OK;
    if (!(f->xwidth > 0.0f && f->xwidth <= 16.0f && f->ywidth > 0.0f && f->ywidth <= 16.0f))
        return fail(RB2_EINVAL, "filter half-widths must be in (0, 16]");
    if (f->kind == RB2_FILTER_GAUSSIAN && !(f->alpha > 0.0f && std::isfinite(f->alpha)))
        return fail(RB2_EINVAL, "Gaussian alpha must be positive");
    return RB2_OK;
}

}  // namespace rb2

extern "C" int rb2_filter_table(const rb2_filter* f, float* table256)
{
    if (!table256) return rb2::fail(RB2_EINVAL, "null table");
    const int rc = rb2::validate_filter(f);
    if (rc) return rc;
    for (int y = 0; y < 16; ++y) {
        const float fy = ((float)y + 0.5f) * f->ywidth / 16.0f;
        for (int x = 0; x < 16; ++x) {
            const float fx = ((float)x + 0.5f) * f->xwidth / 16.0f;
            table256[y * 16 + x] = eval_filter(*f, fx, fy);
        }
    }
    return RB2_OK;
}
