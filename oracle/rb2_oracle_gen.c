/*
 * TEST INFRASTRUCTURE ONLY -- the oracle's copy of the synthetic workload.
 *
 * The batching workload (64 heightfield scenes, incoherent surface rays) is
 * defined by its generator, not by any file of the reference.  The CPU
 * reference arm of the benchmark must build and trace that workload without
 * loading the product library, so this file restates the generator in plain
 * C with the same operations in the same order (compiled with
 * -ffp-contract=off, as the product's host code is): the heightfield is a
 * 4-octave value noise over the unit square (2 triangles per cell) plus
 * axis-aligned boxes; rays start at area-weighted surface points offset along
 * the geometric normal and point in cosine-distributed directions about it.
 * A CPU test checks every output word against the product generator.
 *
 *   PCG32: O'Neill 2014 (pcg32_srandom_r / pcg32_random_r); uniform floats
 *          are (next >> 8) * 2^-24.
 *   Orthonormal basis: Duff et al., "Building an Orthonormal Basis,
 *          Revisited", JCGT 2017.
 */
#include "rb2_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float x, y, z; } g3;

static inline g3 mk3(float x, float y, float z) { g3 r = {x, y, z}; return r; }
static inline g3 add3(g3 a, g3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline g3 sub3(g3 a, g3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline g3 mul3(g3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline float dot3(g3 a, g3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline g3 cross3(g3 a, g3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline g3 norm3(g3 v) { float inv = 1.0f / sqrtf(dot3(v, v)); return mul3(v, inv); }

static inline float gen_uniform(rb2o_pcg32* r) { return (float)(rb2o_pcg32_next(r) >> 8) * (1.0f / 16777216.0f); }
static inline float gen_range(rb2o_pcg32* r, float a, float b) { return a + (b - a) * gen_uniform(r); }

#define NOISE_OCTAVES 4

typedef struct {
    float* lat[NOISE_OCTAVES];
    int res[NOISE_OCTAVES];
} value_noise;

static int noise_init(value_noise* n, uint64_t seed)
{
    for (int o = 0; o < NOISE_OCTAVES; o++) {
        n->res[o] = 4 << o;
        const int w = n->res[o] + 1;
        n->lat[o] = (float*)malloc(sizeof(float) * (size_t)w * w);
        if (!n->lat[o]) return -1;
        rb2o_pcg32 r;
        rb2o_pcg32_seed(&r, seed, 100 + (uint64_t)o);
        for (int k = 0; k < w * w; k++) n->lat[o][k] = gen_range(&r, -1.0f, 1.0f);
    }
    return 0;
}

static void noise_free(value_noise* n)
{
    for (int o = 0; o < NOISE_OCTAVES; o++) free(n->lat[o]);
}

static inline float smooth_step(float t) { return t * t * (3.0f - 2.0f * t); }

static float noise_eval(const value_noise* n, float x, float z)
{
    float sum = 0.0f, norm = 0.0f, amp = 1.0f;
    for (int o = 0; o < NOISE_OCTAVES; o++) {
        const int res = n->res[o];
        float fx = x * (float)res, fz = z * (float)res;
        int ix = (int)fx, iz = (int)fz;
        if (ix < 0) ix = 0;
        if (iz < 0) iz = 0;
        if (ix > res - 1) ix = res - 1;
        if (iz > res - 1) iz = res - 1;
        float tx = smooth_step(fx - (float)ix), tz = smooth_step(fz - (float)iz);
        const float* L = n->lat[o];
        const int w = res + 1;
        float a = L[iz * w + ix], b = L[iz * w + ix + 1], c = L[(iz + 1) * w + ix], d = L[(iz + 1) * w + ix + 1];
        float v = (a + (b - a) * tx) + ((c + (d - c) * tx) - (a + (b - a) * tx)) * tz;
        sum += amp * v;
        norm += amp;
        amp *= 0.5f;
    }
    return sum / norm;
}

int rb2o_gen_heightfield_counts(uint32_t grid_n, uint32_t n_boxes, uint32_t* nv, uint32_t* ntri)
{
    if (!nv || !ntri || grid_n == 0 || grid_n > 16384) return -1;
    *nv = (grid_n + 1) * (grid_n + 1) + 8 * n_boxes;
    *ntri = 2 * grid_n * grid_n + 12 * n_boxes;
    return 0;
}

int rb2o_gen_heightfield(uint64_t seed, uint32_t grid_n, float amplitude, uint32_t n_boxes, float box_min,
                         float box_max, float* v, uint32_t* idx)
{
    if (!v || !idx || grid_n == 0 || grid_n > 16384) return -1;
    value_noise noise;
    memset(&noise, 0, sizeof(noise));
    if (noise_init(&noise, seed)) { noise_free(&noise); return -2; }
    const uint32_t n = grid_n;
    uint32_t nv = 0, nt = 0;
    for (uint32_t j = 0; j <= n; j++)
        for (uint32_t i = 0; i <= n; i++) {
            float x = (float)i / (float)n, z = (float)j / (float)n;
            v[3 * nv + 0] = x;
            v[3 * nv + 1] = amplitude * noise_eval(&noise, x, z);
            v[3 * nv + 2] = z;
            nv++;
        }
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t i = 0; i < n; i++) {
            uint32_t v00 = j * (n + 1) + i, v10 = v00 + 1, v01 = v00 + (n + 1), v11 = v01 + 1;
            idx[3 * nt + 0] = v00; idx[3 * nt + 1] = v01; idx[3 * nt + 2] = v11; nt++;
            idx[3 * nt + 0] = v00; idx[3 * nt + 1] = v11; idx[3 * nt + 2] = v10; nt++;
        }
    /* Boxes: 8 corners (bit 0 = x, bit 1 = y, bit 2 = z), two triangles per face. */
    static const int face[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    rb2o_pcg32 r;
    rb2o_pcg32_seed(&r, seed, 7);
    for (uint32_t b = 0; b < n_boxes; b++) {
        float ex = gen_range(&r, box_min, box_max), ey = gen_range(&r, box_min, box_max);
        float ez = gen_range(&r, box_min, box_max);
        float cx = gen_range(&r, 0.05f, 0.95f), cz = gen_range(&r, 0.05f, 0.95f);
        float base = amplitude * noise_eval(&noise, cx, cz) + gen_range(&r, 0.0f, 0.05f);
        g3 lo = mk3(cx - 0.5f * ex, base, cz - 0.5f * ez), hi = mk3(cx + 0.5f * ex, base + ey, cz + 0.5f * ez);
        uint32_t b0 = nv;
        for (int k = 0; k < 8; k++) {
            v[3 * nv + 0] = (k & 1) ? hi.x : lo.x;
            v[3 * nv + 1] = (k & 2) ? hi.y : lo.y;
            v[3 * nv + 2] = (k & 4) ? hi.z : lo.z;
            nv++;
        }
        for (int f = 0; f < 6; f++) {
            uint32_t a = b0 + face[f][0], c1 = b0 + face[f][1], c2 = b0 + face[f][2], d = b0 + face[f][3];
            idx[3 * nt + 0] = a; idx[3 * nt + 1] = c1; idx[3 * nt + 2] = c2; nt++;
            idx[3 * nt + 0] = a; idx[3 * nt + 1] = c2; idx[3 * nt + 2] = d; nt++;
        }
    }
    noise_free(&noise);
    return 0;
}

/* First index k with cdf[k] > u (upper bound), cdf non-decreasing. */
static uint32_t upper_bound_d(const double* cdf, uint32_t n, double u)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

int rb2o_gen_surface_rays(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, uint64_t seed,
                          uint64_t n_rays, float offset_scale, float anyhit_fraction, float* rays, uint8_t* flags)
{
    if (!v_xyz || !idx3 || !rays || ntri == 0) return -1;
    const g3* V = (const g3*)v_xyz;
    double* cdf = (double*)malloc(sizeof(double) * ntri);
    if (!cdf) return -2;
    double acc = 0.0;
    g3 lo = mk3(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint32_t t = 0; t < ntri; t++) {
        if (idx3[3 * t] >= nv || idx3[3 * t + 1] >= nv || idx3[3 * t + 2] >= nv) { free(cdf); return -1; }
        g3 a = V[idx3[3 * t]], b = V[idx3[3 * t + 1]], c = V[idx3[3 * t + 2]];
        g3 cr = cross3(sub3(b, a), sub3(c, a));
        acc += 0.5 * sqrt((double)dot3(cr, cr));
        cdf[t] = acc;
        const g3 p[3] = {a, b, c};
        for (int k = 0; k < 3; k++) {
            lo.x = p[k].x < lo.x ? p[k].x : lo.x; lo.y = p[k].y < lo.y ? p[k].y : lo.y;
            lo.z = p[k].z < lo.z ? p[k].z : lo.z;
            hi.x = p[k].x > hi.x ? p[k].x : hi.x; hi.y = p[k].y > hi.y ? p[k].y : hi.y;
            hi.z = p[k].z > hi.z ? p[k].z : hi.z;
        }
    }
    if (!(acc > 0.0)) { free(cdf); return -1; }
    g3 diag = sub3(hi, lo);
    const float off = offset_scale * sqrtf(dot3(diag, diag));
    const uint64_t chunk = 1 << 16;
    const int64_t n_chunks = (int64_t)((n_rays + chunk - 1) / chunk);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t ci = 0; ci < n_chunks; ci++) {
        rb2o_pcg32 r;
        rb2o_pcg32_seed(&r, seed, 1000 + (uint64_t)ci);
        uint64_t b = (uint64_t)ci * chunk, e = b + chunk < n_rays ? b + chunk : n_rays;
        for (uint64_t i = b; i < e; i++) {
            double u = (double)gen_uniform(&r) * acc;
            uint32_t t = upper_bound_d(cdf, ntri, u);
            if (t >= ntri) t = ntri - 1;
            g3 a = V[idx3[3 * t]], bb = V[idx3[3 * t + 1]], c = V[idx3[3 * t + 2]];
            float su = sqrtf(gen_uniform(&r)), s2 = gen_uniform(&r);
            float w0 = 1.0f - su, w1 = s2 * su;
            g3 p = add3(add3(mul3(a, w0), mul3(bb, w1)), mul3(c, 1.0f - w0 - w1));
            g3 ng = cross3(sub3(bb, a), sub3(c, a));
            float len2 = dot3(ng, ng);
            ng = len2 > 0.0f ? mul3(ng, 1.0f / sqrtf(len2)) : mk3(0.0f, 1.0f, 0.0f);
            float sign = copysignf(1.0f, ng.z);
            float aa = -1.0f / (sign + ng.z), bq = ng.x * ng.y * aa;
            g3 tx = mk3(1.0f + sign * ng.x * ng.x * aa, sign * bq, -sign * ng.x);
            g3 ty = mk3(bq, sign + ng.y * ng.y * aa, -ng.y);
            float u1 = gen_uniform(&r), u2 = gen_uniform(&r);
            float rad = sqrtf(u1), phi = 6.283185307179586f * u2;
            float lx = rad * cosf(phi), ly = rad * sinf(phi);
            float lz2 = 1.0f - u1;
            float lz = sqrtf(lz2 > 0.0f ? lz2 : 0.0f);
            g3 d = norm3(add3(add3(mul3(tx, lx), mul3(ty, ly)), mul3(ng, lz)));
            g3 o = add3(p, mul3(ng, off));
            float* dst = rays + 8 * i;
            dst[0] = o.x; dst[1] = o.y; dst[2] = o.z; dst[3] = 0.0f;
            dst[4] = d.x; dst[5] = d.y; dst[6] = d.z; dst[7] = FLT_MAX;
            float fsel = gen_uniform(&r);
            if (flags) flags[i] = fsel < anyhit_fraction ? 1 : 0;
        }
    }
    free(cdf);
    return 0;
}
