// Seeded synthetic scenes and ray sets.  See include/rb2_scene.h.
#include "rb2_internal.h"
#include "rb2_scene.h"

#include <algorithm>
#include <atomic>
#include <thread>

namespace rb2 {
namespace {

// PCG32, O'Neill 2014 (pcg32_srandom_r / pcg32_random_r).
struct Pcg32 {
    uint64_t state = 0, inc = 1;
    Pcg32(uint64_t seed, uint64_t stream)
    {
        inc = (stream << 1u) | 1u;
        next();
        state += seed;
        next();
    }
    uint32_t next()
    {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((-rot) & 31));
    }
    float uniform() { return (float)(next() >> 8) * (1.0f / 16777216.0f); }  // [0,1)
    float range(float a, float b) { return a + (b - a) * uniform(); }
};

struct ValueNoise {
    static const int kOctaves = 4;
    std::vector<float> lat[kOctaves];
    int res[kOctaves];
    explicit ValueNoise(uint64_t seed)
    {
        for (int o = 0; o < kOctaves; o++) {
            res[o] = 4 << o;
            Pcg32 r(seed, 100 + o);
            lat[o].resize((size_t)(res[o] + 1) * (res[o] + 1));
            for (float& x : lat[o]) x = r.range(-1.0f, 1.0f);
        }
    }
    static float smooth(float t) { return t * t * (3.0f - 2.0f * t); }
    float operator()(float x, float z) const
    {
        float sum = 0.0f, norm = 0.0f, amp = 1.0f;
        for (int o = 0; o < kOctaves; o++) {
            float fx = x * (float)res[o], fz = z * (float)res[o];
            int ix = std::min(res[o] - 1, std::max(0, (int)fx));
            int iz = std::min(res[o] - 1, std::max(0, (int)fz));
            float tx = smooth(fx - (float)ix), tz = smooth(fz - (float)iz);
            const float* L = lat[o].data();
            int w = res[o] + 1;
            float a = L[iz * w + ix], b = L[iz * w + ix + 1], c = L[(iz + 1) * w + ix], d = L[(iz + 1) * w + ix + 1];
            float v = (a + (b - a) * tx) + ((c + (d - c) * tx) - (a + (b - a) * tx)) * tz;
            sum += amp * v;
            norm += amp;
            amp *= 0.5f;
        }
        return sum / norm;
    }
};

struct MeshOut {
    float* v;
    uint32_t* idx;
    uint32_t* mat;
    uint32_t nv = 0, nt = 0;
    uint32_t add_vertex(f3 p)
    {
        v[3 * nv + 0] = p.x; v[3 * nv + 1] = p.y; v[3 * nv + 2] = p.z;
        return nv++;
    }
    void add_tri(uint32_t a, uint32_t b, uint32_t c, uint32_t m)
    {
        idx[3 * nt + 0] = a; idx[3 * nt + 1] = b; idx[3 * nt + 2] = c;
        if (mat) mat[nt] = m;
        nt++;
    }
};

// Axis-aligned box with outward-facing triangles.
void add_box(MeshOut& m, f3 lo, f3 hi, uint32_t mat, bool inward = false)
{
    uint32_t b = m.nv;
    for (int k = 0; k < 8; k++)
        m.add_vertex(mk((k & 1) ? hi.x : lo.x, (k & 2) ? hi.y : lo.y, (k & 4) ? hi.z : lo.z));
    // Faces as (a,b,c,d) counter-clockwise seen from outside.
    const int f[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    for (int i = 0; i < 6; i++) {
        uint32_t a = b + f[i][0], c1 = b + f[i][1], c2 = b + f[i][2], d = b + f[i][3];
        if (!inward) { m.add_tri(a, c1, c2, mat); m.add_tri(a, c2, d, mat); }
        else { m.add_tri(a, c2, c1, mat); m.add_tri(a, d, c2, mat); }
    }
}

// Grid-tessellated quad: origin + s*ea + t*eb, s,t in [0,1], facing cross(ea, eb).
void add_grid_quad(MeshOut& m, f3 o, f3 ea, f3 eb, uint32_t g, uint32_t mat)
{
    uint32_t base = m.nv;
    for (uint32_t j = 0; j <= g; j++)
        for (uint32_t i = 0; i <= g; i++)
            m.add_vertex(o + ea * ((float)i / (float)g) + eb * ((float)j / (float)g));
    for (uint32_t j = 0; j < g; j++)
        for (uint32_t i = 0; i < g; i++) {
            uint32_t a = base + j * (g + 1) + i, b = a + 1, c = a + (g + 1) + 1, d = a + (g + 1);
            m.add_tri(a, b, c, mat);
            m.add_tri(a, c, d, mat);
        }
}

void add_icosphere(MeshOut& m, f3 c, float r, uint32_t subdiv, uint32_t mat)
{
    const float t = 1.6180339887498949f;
    f3 v[12] = {mk(-1, t, 0), mk(1, t, 0), mk(-1, -t, 0), mk(1, -t, 0), mk(0, -1, t), mk(0, 1, t),
                mk(0, -1, -t), mk(0, 1, -t), mk(t, 0, -1), mk(t, 0, 1), mk(-t, 0, -1), mk(-t, 0, 1)};
    const int f[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                          {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                          {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    std::vector<f3> tris;
    for (auto& face : f) {
        tris.push_back(normalize(v[face[0]]));
        tris.push_back(normalize(v[face[1]]));
        tris.push_back(normalize(v[face[2]]));
    }
    for (uint32_t s = 0; s < subdiv; s++) {
        std::vector<f3> nt;
        nt.reserve(tris.size() * 4);
        for (size_t i = 0; i < tris.size(); i += 3) {
            f3 a = tris[i], b = tris[i + 1], cc = tris[i + 2];
            f3 ab = normalize(a + b), bc = normalize(b + cc), ca = normalize(cc + a);
            f3 q[12] = {a, ab, ca, ab, b, bc, ca, bc, cc, ab, bc, ca};
            nt.insert(nt.end(), q, q + 12);
        }
        tris.swap(nt);
    }
    for (size_t i = 0; i < tris.size(); i += 3) {
        uint32_t a = m.add_vertex(c + tris[i] * r);
        uint32_t b = m.add_vertex(c + tris[i + 1] * r);
        uint32_t d = m.add_vertex(c + tris[i + 2] * r);
        m.add_tri(a, b, d, mat);
    }
}

uint32_t room_wall_grid(uint32_t n_spheres, uint32_t subdiv)
{
    (void)subdiv;
    // Walls are tessellated so that the room carries a fixed share of the
    // triangle budget; larger sphere sets get proportionally finer walls.
    double target = 0.36 * (double)n_spheres * 20.0 * 16.0 / 0.64 / 12.0;
    uint32_t g = (uint32_t)std::max(1.0, std::floor(std::sqrt(target)));
    return std::min<uint32_t>(g, 2048);
}

}  // namespace
}  // namespace rb2

using namespace rb2;

extern "C" {

int rb2_gen_heightfield_counts(uint32_t grid_n, uint32_t n_boxes, uint32_t* nv, uint32_t* ntri)
{
    if (!nv || !ntri || grid_n == 0 || grid_n > 16384) return fail(RB2_EINVAL, "bad heightfield size");
    *nv = (grid_n + 1) * (grid_n + 1) + 8 * n_boxes;
    *ntri = 2 * grid_n * grid_n + 12 * n_boxes;
    return RB2_OK;
}

int rb2_gen_heightfield(uint64_t seed, uint32_t grid_n, float amplitude, uint32_t n_boxes, float box_min,
                        float box_max, float* v_xyz, uint32_t* idx3)
{
    if (!v_xyz || !idx3 || grid_n == 0 || grid_n > 16384) return fail(RB2_EINVAL, "bad heightfield arguments");
    ValueNoise noise(seed);
    MeshOut m{v_xyz, idx3, nullptr};
    const uint32_t n = grid_n;
    for (uint32_t j = 0; j <= n; j++)
        for (uint32_t i = 0; i <= n; i++) {
            float x = (float)i / (float)n, z = (float)j / (float)n;
            m.add_vertex(mk(x, amplitude * noise(x, z), z));
        }
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t i = 0; i < n; i++) {
            uint32_t v00 = j * (n + 1) + i, v10 = v00 + 1, v01 = v00 + (n + 1), v11 = v01 + 1;
            m.add_tri(v00, v01, v11, 0);  // up-facing
            m.add_tri(v00, v11, v10, 0);
        }
    Pcg32 r(seed, 7);
    for (uint32_t b = 0; b < n_boxes; b++) {
        float ex = r.range(box_min, box_max), ey = r.range(box_min, box_max), ez = r.range(box_min, box_max);
        float cx = r.range(0.05f, 0.95f), cz = r.range(0.05f, 0.95f);
        float base = amplitude * noise(cx, cz) + r.range(0.0f, 0.05f);
        add_box(m, mk(cx - 0.5f * ex, base, cz - 0.5f * ez), mk(cx + 0.5f * ex, base + ey, cz + 0.5f * ez), 0);
    }
    return RB2_OK;
}

int rb2_gen_room_counts(uint32_t n_boxes, uint32_t n_spheres, uint32_t sphere_subdiv, uint32_t n_lights, uint32_t* nv,
                        uint32_t* ntri)
{
    if (!nv || !ntri || sphere_subdiv > 6) return fail(RB2_EINVAL, "bad room arguments");
    uint32_t g = room_wall_grid(n_spheres, sphere_subdiv);
    uint64_t per_sphere = 20ull << (2 * sphere_subdiv);
    uint64_t t = 6ull * 2 * g * g + 12ull * n_boxes + per_sphere * n_spheres + 2ull * n_lights;
    uint64_t v = 6ull * (g + 1) * (g + 1) + 8ull * n_boxes + 3 * per_sphere * n_spheres + 4ull * n_lights;
    if (t > 0xFFFFFFF0ull || v > 0xFFFFFFF0ull) return fail(RB2_EINVAL, "room too large");
    *ntri = (uint32_t)t;
    *nv = (uint32_t)v;
    return RB2_OK;
}

int rb2_gen_room(uint64_t seed, uint32_t n_boxes, uint32_t n_spheres, uint32_t sphere_subdiv, float rmin, float rmax,
                 uint32_t n_lights, float* v_xyz, uint32_t* idx3, uint32_t* tri_material)
{
    if (!v_xyz || !idx3 || !tri_material || sphere_subdiv > 6 || !(rmin > 0.0f) || rmax < rmin)
        return fail(RB2_EINVAL, "bad room arguments");
    MeshOut m{v_xyz, idx3, tri_material};
    uint32_t g = room_wall_grid(n_spheres, sphere_subdiv);
    // Inward-facing walls: material ids 0..5.
    add_grid_quad(m, mk(0, 0, 0), mk(0, 0, 1), mk(1, 0, 0), g, 0);   // floor, normal +y
    add_grid_quad(m, mk(0, 1, 0), mk(1, 0, 0), mk(0, 0, 1), g, 1);   // ceiling, normal -y
    add_grid_quad(m, mk(0, 0, 0), mk(0, 1, 0), mk(0, 0, 1), g, 2);   // x=0 wall, normal +x
    add_grid_quad(m, mk(1, 0, 0), mk(0, 0, 1), mk(0, 1, 0), g, 3);   // x=1 wall, normal -x
    add_grid_quad(m, mk(0, 0, 0), mk(1, 0, 0), mk(0, 1, 0), g, 4);   // z=0 wall, normal +z
    add_grid_quad(m, mk(0, 0, 1), mk(0, 1, 0), mk(1, 0, 0), g, 5);   // z=1 wall, normal -z
    uint32_t mat = 6;
    Pcg32 rb(seed, 11);
    for (uint32_t b = 0; b < n_boxes; b++) {
        float ex = rb.range(0.03f, 0.15f), ey = rb.range(0.03f, 0.3f), ez = rb.range(0.03f, 0.15f);
        float cx = rb.range(0.1f, 0.9f), cz = rb.range(0.1f, 0.9f);
        add_box(m, mk(cx - 0.5f * ex, 0.0f, cz - 0.5f * ez), mk(cx + 0.5f * ex, ey, cz + 0.5f * ez), mat++);
    }
    Pcg32 rs(seed, 13);
    const float lr = std::log(rmin), hr = std::log(rmax);
    for (uint32_t s = 0; s < n_spheres; s++) {
        float r = std::exp(rs.range(lr, hr));
        r = std::min(r, 0.45f);
        f3 c = mk(rs.range(r, 1.0f - r), rs.range(r, 0.85f - r > r ? 0.85f - r : r), rs.range(r, 1.0f - r));
        add_icosphere(m, c, r, sphere_subdiv, mat++);
    }
    // Emitters: downward-facing quads just below the ceiling.
    for (uint32_t l = 0; l < n_lights; l++) {
        float cx = n_lights == 1 ? 0.5f : 0.25f + 0.5f * (float)l / (float)(n_lights - 1);
        float s = 0.1f;
        f3 o = mk(cx - s, 0.995f, 0.5f - s);
        uint32_t a = m.add_vertex(o), b = m.add_vertex(o + mk(2 * s, 0, 0));
        uint32_t c = m.add_vertex(o + mk(2 * s, 0, 2 * s)), d = m.add_vertex(o + mk(0, 0, 2 * s));
        // cross(b-a, d-a) = (+x) x (+z) = -y: facing down into the room.
        m.add_tri(a, b, d, mat);
        m.add_tri(b, c, d, mat);
        mat++;
    }
    return RB2_OK;
}

int rb2_gen_surface_rays(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, uint64_t seed,
                         uint64_t n_rays, float offset_scale, float anyhit_fraction, float* rays, uint8_t* flags)
{
    if (!v_xyz || !idx3 || !rays || ntri == 0) return fail(RB2_EINVAL, "bad ray-generation arguments");
    const f3* V = reinterpret_cast<const f3*>(v_xyz);
    std::vector<double> cdf(ntri);
    double acc = 0.0;
    Box sb;
    for (uint32_t t = 0; t < ntri; t++) {
        if (idx3[3 * t] >= nv || idx3[3 * t + 1] >= nv || idx3[3 * t + 2] >= nv) return fail(RB2_EINVAL, "index out of range");
        f3 a = V[idx3[3 * t]], b = V[idx3[3 * t + 1]], c = V[idx3[3 * t + 2]];
        f3 cr = cross(b - a, c - a);
        acc += 0.5 * std::sqrt((double)dot(cr, cr));
        cdf[t] = acc;
        sb.insert(a); sb.insert(b); sb.insert(c);
    }
    if (!(acc > 0.0)) return fail(RB2_EINVAL, "scene has zero area");
    f3 diag = sb.hi - sb.lo;
    const float off = offset_scale * std::sqrt(dot(diag, diag));
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t chunk = 1 << 16;
    const uint64_t n_chunks = (n_rays + chunk - 1) / chunk;
    std::atomic<uint64_t> next{0};
    auto work = [&] {
        for (;;) {
            uint64_t ci = next++;
            if (ci >= n_chunks) break;
            Pcg32 r(seed, 1000 + ci);
            uint64_t b = ci * chunk, e = std::min(n_rays, b + chunk);
            for (uint64_t i = b; i < e; i++) {
                double u = (double)r.uniform() * acc;
                uint32_t t = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
                if (t >= ntri) t = ntri - 1;
                f3 a = V[idx3[3 * t]], bb = V[idx3[3 * t + 1]], c = V[idx3[3 * t + 2]];
                float su = std::sqrt(r.uniform()), s2 = r.uniform();
                float w0 = 1.0f - su, w1 = s2 * su;
                f3 p = a * w0 + bb * w1 + c * (1.0f - w0 - w1);
                f3 ng = cross(bb - a, c - a);
                float len2 = dot(ng, ng);
                ng = len2 > 0.0f ? ng * (1.0f / std::sqrt(len2)) : mk(0, 1, 0);
                // Orthonormal basis (Duff et al., "Building an Orthonormal Basis, Revisited", JCGT 2017).
                float sign = std::copysign(1.0f, ng.z);
                float aa = -1.0f / (sign + ng.z), bq = ng.x * ng.y * aa;
                f3 tx = mk(1.0f + sign * ng.x * ng.x * aa, sign * bq, -sign * ng.x);
                f3 ty = mk(bq, sign + ng.y * ng.y * aa, -ng.y);
                float u1 = r.uniform(), u2 = r.uniform();
                float rad = std::sqrt(u1), phi = 6.283185307179586f * u2;
                float lx = rad * std::cos(phi), ly = rad * std::sin(phi), lz = std::sqrt(std::max(0.0f, 1.0f - u1));
                f3 d = normalize(tx * lx + ty * ly + ng * lz);
                f3 o = p + ng * off;
                float* dst = rays + 8 * i;
                dst[0] = o.x; dst[1] = o.y; dst[2] = o.z; dst[3] = 0.0f;
                dst[4] = d.x; dst[5] = d.y; dst[6] = d.z; dst[7] = FLT_MAX;
                float fsel = r.uniform();
                if (flags) flags[i] = fsel < anyhit_fraction ? 1 : 0;
            }
        }
    };
    std::vector<std::thread> th;
    for (unsigned k = 1; k < nt; k++) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
    return RB2_OK;
}

int rb2_pcg32_fill(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out)
{
    if (!out) return fail(RB2_EINVAL, "null output");
    Pcg32 r(seed, stream);
    for (uint32_t i = 0; i < n; i++) out[i] = r.next();
    return RB2_OK;
}

}  // extern "C"
