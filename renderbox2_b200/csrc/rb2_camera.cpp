// Perspective camera set-up (host).  Restates the transform algebra of the
// reference's PerspectiveCamera (core/camera.cu:30-56) and Transform helpers
// (core/transform.cu:81-126, core/transform.h:205-333) with the same
// operation order, so the matrices handed to the device ray generator are
// bit-identical to the reference's and so are the rays.
#include "rb2_internal.h"
#include "rb2_render.h"

namespace rb2 {

void invert4_public(const float m[16], float out[16]);

namespace {

struct M4 {
    float m[16];
    static M4 identity()
    {
        M4 r;
        for (int i = 0; i < 16; i++) r.m[i] = (i % 5 == 0) ? 1.0f : 0.0f;
        return r;
    }
    M4 operator*(const M4& b) const
    {
        M4 r;
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
                r.m[i * 4 + j] = m[i * 4 + 0] * b.m[0 * 4 + j] + m[i * 4 + 1] * b.m[1 * 4 + j] +
                                 m[i * 4 + 2] * b.m[2 * 4 + j] + m[i * 4 + 3] * b.m[3 * 4 + j];
        return r;
    }
    M4 inverse() const
    {
        M4 r;
        invert4_public(m, r.m);
        return r;
    }
};

struct Xform {
    M4 m, inv;
    explicit Xform(const M4& a) : m(a), inv(a.inverse()) {}
    Xform(const M4& a, const M4& b) : m(a), inv(b) {}
    Xform operator*(const Xform& t) const { return Xform(m * t.m, t.inv * inv); }
    Xform inverse() const { return Xform(inv, m); }
};

Xform scale(float sx, float sy, float sz)
{
    M4 r = M4::identity();
    r.m[0] = sx; r.m[5] = sy; r.m[10] = sz; r.m[15] = 1.0f;
    return Xform(r);
}

Xform translate(float x, float y, float z)
{
    M4 r = M4::identity();
    r.m[3] = x; r.m[7] = y; r.m[11] = z;
    return Xform(r);
}

Xform lookat(f3 pos, f3 look, f3 up)
{
    M4 c;
    c.m[3] = pos.x; c.m[7] = pos.y; c.m[11] = pos.z; c.m[15] = 1.0f;
    f3 dir = normalize(look - pos);
    f3 left = normalize(cross(normalize(up), dir));
    f3 nu = cross(dir, left);
    c.m[0] = left.x; c.m[4] = left.y; c.m[8] = left.z; c.m[12] = 0.0f;
    c.m[1] = nu.x; c.m[5] = nu.y; c.m[9] = nu.z; c.m[13] = 0.0f;
    c.m[2] = dir.x; c.m[6] = dir.y; c.m[10] = dir.z; c.m[14] = 0.0f;
    return Xform(c.inverse(), c);
}

Xform perspective(float fov, float n, float f)
{
    M4 p;
    const float vals[16] = {1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f,
                            0.0f, 0.0f, f / (f - n), -f * n / (f - n), 0.0f, 0.0f, 1.0f, 0.0f};
    for (int i = 0; i < 16; i++) p.m[i] = vals[i];
    const float pi_f = 3.14159265358979323846f;
    float rad = (pi_f / 180.f) * fov;
    float inv_tan = 1.0f / tanf(rad / 2.0f);
    return scale(inv_tan, inv_tan, 1.0f) * Xform(p);
}

}  // namespace
}  // namespace rb2

using namespace rb2;

extern "C" int rb2_camera_init(rb2_camera* cam, const float eye[3], const float look[3], const float up[3],
                               uint32_t width, uint32_t height, float fov_deg)
{
    if (!cam || !eye || !look || !up || width == 0 || height == 0 || !(fov_deg > 0.0f && fov_deg < 180.0f))
        return fail(RB2_EINVAL, "bad camera arguments");
    f3 e = mk(eye[0], eye[1], eye[2]), l = mk(look[0], look[1], look[2]), u = mk(up[0], up[1], up[2]);
    Xform world_to_camera = lookat(e, l, u) * scale(-1.0f, 1.0f, 1.0f);
    Xform camera_to_world = world_to_camera.inverse();
    Xform cam_to_screen = perspective(fov_deg, 1.0f, 1000.0f);
    Xform screen_to_raster = scale((float)width, (float)height, 1.0f) * scale(0.5f, -0.5f, 1.0f) *
                             translate(1.0f, -1.0f, 0.0f);
    Xform raster_to_screen = screen_to_raster.inverse();
    Xform raster_to_camera = cam_to_screen.inverse() * raster_to_screen;
    for (int i = 0; i < 16; i++) {
        cam->raster_to_camera[i] = raster_to_camera.m.m[i];
        cam->camera_to_world[i] = camera_to_world.m.m[i];
    }
    cam->width = width;
    cam->height = height;
    for (int k = 0; k < 3; k++) { cam->eye[k] = eye[k]; cam->lookat[k] = look[k]; cam->up[k] = up[k]; }
    cam->fov_deg = fov_deg;
    return RB2_OK;
}
