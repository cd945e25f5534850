/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  See rb2_oracle.h.
 *
 * Arithmetic specification (the product kernel implements the same operations
 * with __fmaf_rn / __fmul_rn / IEEE division, so results are bit-identical):
 *
 *   ray setup   (cuda_tracer_functions.cu:78-84)
 *     idir_c = 1.0f / (|d_c| > 2^-80 ? d_c : copysign(2^-80, d_c))   IEEE div
 *     ood_c  = o_c * idir_c                                          RN mul
 *   slab        (cuda_tracer_functions.cu:103-118)
 *     s = fmaf(bound, idir_c, -ood_c)       (nvcc contracts  b*idir - ood)
 *   spans       (cudatracerkernels.h:213-256; PTX vmin/vmax are exact integer ops)
 *     cmin = imax{ fmin(lox,hix), fmin(loy,hiy), imin(loz,hiz), tmin }
 *     cmax = imin{ fmax(lox,hix), fmax(loy,hiy), imax(loz,hiz), hitT }
 *     imin/imax compare the float bit patterns as signed 32-bit integers;
 *     fmin(a,b) = (a < b) ? a : b,  fmax(a,b) = (a > b) ? a : b
 *   Woop test   (cuda_tracer_functions.cu:188-208)
 *     Oz = fma(-oz,w0.z, fma(-oy,w0.y, fma(-ox,w0.x, w0.w)))
 *     Dz = fma(dz,w0.z, fma(dy,w0.y, dx*w0.x));  t = Oz * (1.0f / Dz)
 *     accept t if tmin < t < hitT
 *     u  = fma(t, Dx, Ox) with Ox = fma(oz,w1.z, fma(oy,w1.y, fma(ox,w1.x, w1.w))),
 *          Dx = fma(dz,w1.z, fma(dy,w1.y, dx*w1.x));  need u >= 0
 *     v  = same with w2;  need v >= 0 and (u + v) <= 1
 *
 * Traversal order is the reference's while-while loop run by one lane: the
 * warp vote "no lane still has an unpostponed slot" reduces to "this lane has
 * postponed a leaf", so each leaf is processed as soon as it is found (two
 * when both children of a node are leaves).  u, v are reported for the
 * accepted triangle.  Counts: nodes = inner-node fetches, tris = Woop
 * triangle fetches, leafterms = leaf terminator fetches.
 */
#include "rb2_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RB2O_SENTINEL 0x76543210
#define RB2O_STACK 64
#define RB2O_PI 3.14159265358979323846

static inline float as_f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline int32_t as_i(float f) { int32_t i; memcpy(&i, &f, 4); return i; }
static inline float i_as_f(int32_t i) { float f; memcpy(&f, &i, 4); return f; }

static inline float fmin_s(float a, float b) { return (a < b) ? a : b; }
static inline float fmax_s(float a, float b) { return (a > b) ? a : b; }
static inline float imin_f(float a, float b) { int32_t x = as_i(a), y = as_i(b); return i_as_f(x < y ? x : y); }
static inline float imax_f(float a, float b) { int32_t x = as_i(a), y = as_i(b); return i_as_f(x > y ? x : y); }

static inline float span_begin(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imax_f(imax_f(fmin_s(a0, a1), fmin_s(b0, b1)), imax_f(imin_f(c0, c1), d));
}
static inline float span_end(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imin_f(imin_f(fmax_s(a0, a1), fmax_s(b0, b1)), imin_f(imax_f(c0, c1), d));
}

typedef struct {
    float ox, oy, oz, dx, dy, dz, idx, idy, idz, oodx, oody, oodz, tmin;
} ray_setup;

static inline void setup_ray(const float* r, ray_setup* s)
{
    const float ooeps = 0x1p-80f;
    s->ox = r[0]; s->oy = r[1]; s->oz = r[2]; s->tmin = r[3];
    s->dx = r[4]; s->dy = r[5]; s->dz = r[6];
    s->idx = 1.0f / (fabsf(s->dx) > ooeps ? s->dx : copysignf(ooeps, s->dx));
    s->idy = 1.0f / (fabsf(s->dy) > ooeps ? s->dy : copysignf(ooeps, s->dy));
    s->idz = 1.0f / (fabsf(s->dz) > ooeps ? s->dz : copysignf(ooeps, s->dz));
    s->oodx = s->ox * s->idx;
    s->oody = s->oy * s->idy;
    s->oodz = s->oz * s->idz;
}

/* Returns 1 when the triangle is accepted; writes t,u,v. */
static inline int woop_accept(const ray_setup* s, const float* w, float hitT, float* tuv)
{
    float Oz = fmaf(-s->oz, w[2], fmaf(-s->oy, w[1], fmaf(-s->ox, w[0], w[3])));
    float Dz = fmaf(s->dz, w[2], fmaf(s->dy, w[1], s->dx * w[0]));
    float invDz = 1.0f / Dz;
    float t = Oz * invDz;
    if (!(t > s->tmin && t < hitT)) return 0;
    float Ox = fmaf(s->oz, w[6], fmaf(s->oy, w[5], fmaf(s->ox, w[4], w[7])));
    float Dx = fmaf(s->dz, w[6], fmaf(s->dy, w[5], s->dx * w[4]));
    float u = fmaf(t, Dx, Ox);
    if (!(u >= 0.0f)) return 0;
    float Oy = fmaf(s->oz, w[10], fmaf(s->oy, w[9], fmaf(s->ox, w[8], w[11])));
    float Dy = fmaf(s->dz, w[10], fmaf(s->dy, w[9], s->dx * w[8]));
    float v = fmaf(t, Dy, Oy);
    if (!(v >= 0.0f && u + v <= 1.0f)) return 0;
    tuv[0] = t; tuv[1] = u; tuv[2] = v;
    return 1;
}

static void trace_one(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx,
                      const float* r, int any_hit, rb2o_hit* out, rb2o_counts* cnt)
{
    ray_setup s;
    setup_ray(r, &s);
    float hitT = r[7];
    int32_t stack[RB2O_STACK + 2];
    int sp = 0;
    stack[0] = RB2O_SENTINEL;
    int32_t leafAddr = 0, nodeAddr = 0, hitIndex = -1;
    float hu = 0.0f, hv = 0.0f;
    uint32_t n_nodes = 0, n_tris = 0, n_terms = 0;

    while (nodeAddr != RB2O_SENTINEL) {
        while ((uint32_t)nodeAddr < (uint32_t)RB2O_SENTINEL) {
            const uint32_t* n = nodes + 4 * (size_t)nodeAddr;
            n_nodes++;
            const float n0x0 = as_f(n[0]), n0x1 = as_f(n[1]), n0y0 = as_f(n[2]), n0y1 = as_f(n[3]);
            const float n1x0 = as_f(n[4]), n1x1 = as_f(n[5]), n1y0 = as_f(n[6]), n1y1 = as_f(n[7]);
            const float z00 = as_f(n[8]), z01 = as_f(n[9]), z10 = as_f(n[10]), z11 = as_f(n[11]);
            int32_t c0 = (int32_t)n[12], c1 = (int32_t)n[13];

            const float c0lox = fmaf(n0x0, s.idx, -s.oodx);
            const float c0hix = fmaf(n0x1, s.idx, -s.oodx);
            const float c0loy = fmaf(n0y0, s.idy, -s.oody);
            const float c0hiy = fmaf(n0y1, s.idy, -s.oody);
            const float c0loz = fmaf(z00, s.idz, -s.oodz);
            const float c0hiz = fmaf(z01, s.idz, -s.oodz);
            const float c1loz = fmaf(z10, s.idz, -s.oodz);
            const float c1hiz = fmaf(z11, s.idz, -s.oodz);
            const float c0min = span_begin(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, s.tmin);
            const float c0max = span_end(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, hitT);
            const float c1lox = fmaf(n1x0, s.idx, -s.oodx);
            const float c1hix = fmaf(n1x1, s.idx, -s.oodx);
            const float c1loy = fmaf(n1y0, s.idy, -s.oody);
            const float c1hiy = fmaf(n1y1, s.idy, -s.oody);
            const float c1min = span_begin(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, s.tmin);
            const float c1max = span_end(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, hitT);

            const int swp = (c1min < c0min);
            const int t0 = (c0max >= c0min);
            const int t1 = (c1max >= c1min);
            if (!t0 && !t1) {
                nodeAddr = stack[sp--];
            } else {
                nodeAddr = t0 ? c0 : c1;
                if (t0 && t1) {
                    if (swp) { int32_t tmp = nodeAddr; nodeAddr = c1; c1 = tmp; }
                    stack[++sp] = c1;
                }
            }
            if (nodeAddr < 0 && leafAddr >= 0) {
                leafAddr = nodeAddr;
                nodeAddr = stack[sp--];
            }
            if (!(leafAddr >= 0)) break; /* single-lane warp vote */
        }

        while (leafAddr < 0) {
            for (int32_t triAddr = ~leafAddr;; triAddr += 3) {
                const uint32_t* w = woop + 4 * (size_t)triAddr;
                if (w[0] == 0x80000000u) { n_terms++; break; }
                n_tris++;
                float wf[12];
                for (int k = 0; k < 12; k++) wf[k] = as_f(w[k]);
                float tuv[3];
                if (woop_accept(&s, wf, hitT, tuv)) {
                    hitT = tuv[0]; hu = tuv[1]; hv = tuv[2];
                    hitIndex = triAddr;
                    if (any_hit) { nodeAddr = RB2O_SENTINEL; break; }
                }
            }
            leafAddr = nodeAddr;
            if (nodeAddr < 0) nodeAddr = stack[sp--];
        }
    }

    if (hitIndex >= 0) {
        out->prim = (int32_t)triidx[hitIndex];
        out->t = hitT; out->u = hu; out->v = hv;
    } else {
        out->prim = -1; out->t = r[7]; out->u = 0.0f; out->v = 0.0f;
    }
    if (cnt) { cnt->nodes = n_nodes; cnt->tris = n_tris; cnt->leafterms = n_terms; cnt->pad = 0; }
}

void rb2o_trace(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx,
                const float* rays, uint32_t n, int any_hit, const uint8_t* mask,
                rb2o_hit* out, rb2o_counts* counts, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        if (mask && mask[i] == 0) {
            out[i].prim = -1; out[i].t = rays[8 * i + 7]; out[i].u = 0.0f; out[i].v = 0.0f;
            if (counts) memset(&counts[i], 0, sizeof(rb2o_counts));
            continue;
        }
        trace_one(nodes, woop, triidx, rays + 8 * i, any_hit, out + i, counts ? counts + i : NULL);
    }
    (void)nthreads;
}

void rb2o_isect(const float* verts, const uint32_t* tris4, const float* rays, const rb2o_hit* hits, uint32_t n,
                rb2o_isect_soa* out)
{
    for (uint32_t i = 0; i < n; i++) {
        const rb2o_hit* h = hits + i;
        if (h->prim < 0) { out->intersected[i] = 0; continue; }
        const uint32_t* tr = tris4 + 4 * (size_t)h->prim;
        const float* a = verts + 3 * (size_t)tr[0];
        const float* b = verts + 3 * (size_t)tr[1];
        const float* c = verts + 3 * (size_t)tr[2];
        const float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
        const float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
        const float cx = e1y * e2z - e1z * e2y;
        const float cy = e1z * e2x - e1x * e2z;
        const float cz = e1x * e2y - e1y * e2x;
        const float len2 = (cx * cx + cy * cy) + cz * cz;
        const float inv = 1.0f / sqrtf(len2);
        const float ng[3] = {cx * inv, cy * inv, cz * inv};
        const float* r = rays + 8 * (size_t)i;
        const float t = h->t;
        for (int k = 0; k < 3; k++) {
            out->position[(size_t)k * n + i] = r[k] + r[4 + k] * t;
            out->ng[(size_t)k * n + i] = ng[k];
            out->ns[(size_t)k * n + i] = ng[k];
            out->wi[(size_t)k * n + i] = -r[4 + k];
        }
        const float dn = (ng[0] * r[4] + ng[1] * r[5]) + ng[2] * r[6];
        out->front[i] = dn < 0.0f ? 1 : 0;
        out->uv[2 * (size_t)i] = h->u;
        out->uv[2 * (size_t)i + 1] = h->v;
        out->prim[i] = (uint32_t)h->prim;
        out->material[i] = tr[3];
        out->epsilon[i] = 1.0e-3f * t;
        out->intersected[i] = 1;
    }
}

static float film_eval(uint32_t kind, float xw, float yw, float alpha, float x, float y)
{
    if (kind == 2) return fmaxf(0.0f, xw - fabsf(x)) * fmaxf(0.0f, yw - fabsf(y));
    if (kind == 3) {
        const float ex = expf(-alpha * xw * xw), ey = expf(-alpha * yw * yw);
        return fmaxf(0.0f, expf(-alpha * x * x) - ex) * fmaxf(0.0f, expf(-alpha * y * y) - ey);
    }
    return 1.0f;
}

void rb2o_filter_table(uint32_t kind, float xw, float yw, float alpha, float* table256)
{
    for (int y = 0; y < 16; ++y) {
        const float fy = ((float)y + 0.5f) * yw / 16.0f;
        for (int x = 0; x < 16; ++x) {
            const float fx = ((float)x + 0.5f) * xw / 16.0f;
            table256[y * 16 + x] = film_eval(kind, xw, yw, alpha, fx, fy);
        }
    }
}

void rb2o_film(uint32_t kind, float xw, float yw, float alpha, uint32_t width, uint32_t height, uint32_t spp,
               const float* xy, const float* L4, float* rgb)
{
    const size_t npix = (size_t)width * height;
    if (kind == 0) {
        const float inv = 1.0f / (float)spp;
        for (size_t p = 0; p < npix; p++) {
            float a[3] = {0.0f, 0.0f, 0.0f};
            for (uint32_t j = 0; j < spp; j++)
                for (int c = 0; c < 3; c++) a[c] = a[c] + L4[4 * ((size_t)j * npix + p) + c];
            for (int c = 0; c < 3; c++) rgb[3 * p + c] = a[c] * inv;
        }
        return;
    }
    float table[256];
    rb2o_filter_table(kind, xw, yw, alpha, table);
    const float ixw = 1.0f / xw, iyw = 1.0f / yw;
    /* Candidate source pixels: every pixel whose samples can reach (x, y). */
    const int rx = (int)floorf(xw + 0.5f) + 1, ry = (int)floorf(yw + 0.5f) + 1;
    for (int y = 0; y < (int)height; y++) {
        for (int x = 0; x < (int)width; x++) {
            float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (int qy = y - ry; qy <= y + ry; qy++) {
                if (qy < 0 || qy >= (int)height) continue;
                for (int qx = x - rx; qx <= x + rx; qx++) {
                    if (qx < 0 || qx >= (int)width) continue;
                    const size_t q = (size_t)qy * width + (size_t)qx;
                    for (uint32_t j = 0; j < spp; j++) {
                        const size_t k = (size_t)j * npix + q;
                        const float dx = xy[2 * k] - 0.5f, dy = xy[2 * k + 1] - 0.5f;
                        if (x < (int)ceilf(dx - xw) || x > (int)floorf(dx + xw) || y < (int)ceilf(dy - yw) ||
                            y > (int)floorf(dy + yw))
                            continue;
                        const float fx = fabsf((((float)x - dx) * ixw) * 16.0f);
                        const float fy = fabsf((((float)y - dy) * iyw) * 16.0f);
                        int ix = (int)floorf(fx), iy = (int)floorf(fy);
                        if (ix > 15) ix = 15;
                        if (iy > 15) iy = 15;
                        const float w = table[iy * 16 + ix];
                        for (int c = 0; c < 3; c++) a[c] = a[c] + w * L4[4 * k + c];
                        a[3] = a[3] + w;
                    }
                }
            }
            const float inv = a[3] != 0.0f ? 1.0f / a[3] : 0.0f;
            for (int c = 0; c < 3; c++) rgb[3 * ((size_t)y * width + x) + c] = fmaxf(0.0f, a[c] * inv);
        }
    }
}

int rb2o_woop_test(const uint32_t* woop12, const float* ray8, float tmax, float* tuv)
{
    ray_setup s;
    setup_ray(ray8, &s);
    float wf[12];
    for (int k = 0; k < 12; k++) wf[k] = as_f(woop12[k]);
    return woop_accept(&s, wf, tmax, tuv);
}

void rb2o_bruteforce(const uint32_t* woop, const uint32_t* triidx, uint32_t n_woop_u4,
                     const float* rays, uint32_t n, rb2o_hit* out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        ray_setup s;
        setup_ray(rays + 8 * i, &s);
        float hitT = rays[8 * i + 7];
        int32_t best = -1;
        float bu = 0.0f, bv = 0.0f;
        uint32_t slot = 0;
        while (slot < n_woop_u4) {
            const uint32_t* w = woop + 4 * (size_t)slot;
            if (w[0] == 0x80000000u) { slot += 1; continue; }
            float wf[12];
            for (int k = 0; k < 12; k++) wf[k] = as_f(w[k]);
            float tuv[3];
            if (woop_accept(&s, wf, hitT, tuv)) {
                hitT = tuv[0]; bu = tuv[1]; bv = tuv[2]; best = (int32_t)slot;
            }
            slot += 3;
        }
        if (best >= 0) {
            out[i].prim = (int32_t)triidx[best]; out[i].t = hitT; out[i].u = bu; out[i].v = bv;
        } else {
            out[i].prim = -1; out[i].t = rays[8 * i + 7]; out[i].u = 0.0f; out[i].v = 0.0f;
        }
    }
    (void)nthreads;
}

/* Distinct triangle ids among `ids[0..n)`; appends `id` when new. */
static inline void add_distinct(uint32_t* ids, uint32_t* n, uint32_t cap, uint32_t id)
{
    for (uint32_t k = 0; k < *n; k++)
        if (ids[k] == id) return;
    if (*n < cap) ids[(*n)++] = id;
}

#define RB2O_TIE_CAP 64

void rb2o_tie_count_brute(const uint32_t* woop, const uint32_t* triidx, uint32_t n_woop_u4, const float* rays,
                          uint32_t n, const rb2o_hit* hits, uint32_t* out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        out[i] = 0;
        if (hits[i].prim < 0) continue;
        ray_setup s;
        setup_ray(rays + 8 * i, &s);
        const float t = hits[i].t;
        uint32_t ids[RB2O_TIE_CAP], nid = 0;
        for (uint32_t slot = 0; slot < n_woop_u4;) {
            const uint32_t* w = woop + 4 * (size_t)slot;
            if (w[0] == 0x80000000u) { slot += 1; continue; }
            float wf[12];
            for (int k = 0; k < 12; k++) wf[k] = as_f(w[k]);
            float tuv[3];
            if (woop_accept(&s, wf, FLT_MAX, tuv) && tuv[0] == t) add_distinct(ids, &nid, RB2O_TIE_CAP, triidx[slot]);
            slot += 3;
        }
        out[i] = nid;
    }
    (void)nthreads;
}

void rb2o_tie_count(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx, const float* rays,
                    uint32_t n, const rb2o_hit* hits, uint32_t* out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        out[i] = 0;
        if (hits[i].prim < 0) continue;
        ray_setup s;
        setup_ray(rays + 8 * i, &s);
        const float t = hits[i].t;
        /* Visit every node whose box the ray enters before t plus a slack
         * that covers the slab test's rounding (boxes whose face holds the
         * hit point stay in), and never shrink the interval. */
        const float omax = fmaxf(fabsf(s.ox), fmaxf(fabsf(s.oy), fabsf(s.oz)));
        const float tcut = t + fabsf(t) * 1.0e-3f + (omax + 1.0f) * 1.0e-5f;
        uint32_t ids[RB2O_TIE_CAP], nid = 0;
        int32_t stack[4 * RB2O_STACK];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            int32_t a = stack[--sp];
            if (a < 0) {
                for (int32_t triAddr = ~a;; triAddr += 3) {
                    const uint32_t* w = woop + 4 * (size_t)triAddr;
                    if (w[0] == 0x80000000u) break;
                    float wf[12];
                    for (int k = 0; k < 12; k++) wf[k] = as_f(w[k]);
                    float tuv[3];
                    if (woop_accept(&s, wf, FLT_MAX, tuv) && tuv[0] == t)
                        add_distinct(ids, &nid, RB2O_TIE_CAP, triidx[triAddr]);
                }
                continue;
            }
            const uint32_t* nd = nodes + 4 * (size_t)a;
            const float lo0[3] = {as_f(nd[0]), as_f(nd[2]), as_f(nd[8])};
            const float hi0[3] = {as_f(nd[1]), as_f(nd[3]), as_f(nd[9])};
            const float lo1[3] = {as_f(nd[4]), as_f(nd[6]), as_f(nd[10])};
            const float hi1[3] = {as_f(nd[5]), as_f(nd[7]), as_f(nd[11])};
            const float id3[3] = {s.idx, s.idy, s.idz}, ood3[3] = {s.oodx, s.oody, s.oodz};
            const int32_t ch[2] = {(int32_t)nd[12], (int32_t)nd[13]};
            for (int c = 0; c < 2; c++) {
                const float* lo = c ? lo1 : lo0;
                const float* hi = c ? hi1 : hi0;
                float e[3], x[3];
                for (int k = 0; k < 3; k++) {
                    float p = fmaf(lo[k], id3[k], -ood3[k]), q = fmaf(hi[k], id3[k], -ood3[k]);
                    e[k] = fminf(p, q);
                    x[k] = fmaxf(p, q);
                }
                float cmin = fmaxf(fmaxf(e[0], e[1]), fmaxf(e[2], s.tmin));
                float cmax = fminf(fminf(x[0], x[1]), fminf(x[2], tcut));
                if (cmax >= cmin * (cmin > 0.0f ? 1.0f - 1.0e-5f : 1.0f + 1.0e-5f) && sp < 4 * RB2O_STACK)
                    stack[sp++] = ch[c];
            }
        }
        out[i] = nid;
    }
    (void)nthreads;
}

/* PCG32: O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically
 * Good Algorithms for Random Number Generation" (2014), reference pcg32_random_r. */
void rb2o_pcg32_seed(rb2o_pcg32* r, uint64_t initstate, uint64_t initseq)
{
    r->state = 0u;
    r->inc = (initseq << 1u) | 1u;
    rb2o_pcg32_next(r);
    r->state += initstate;
    rb2o_pcg32_next(r);
}

uint32_t rb2o_pcg32_next(rb2o_pcg32* r)
{
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
}

/* ======================================================================= shading
 * Reference estimators for the integrator tests.  Shading math in double;
 * rays handed to the traversal restatement are rounded to float. */

typedef struct { double x, y, z; } d3;
static inline d3 D3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 dadd(d3 a, d3 b) { return D3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dsub(d3 a, d3 b) { return D3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dmul(d3 a, double s) { return D3(a.x * s, a.y * s, a.z * s); }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b) { return D3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline d3 dnorm(d3 v) { return dmul(v, 1.0 / sqrt(ddot(v, v))); }
static inline d3 vtx(const rb2o_scene* s, uint32_t i) { return D3(s->verts[3 * i], s->verts[3 * i + 1], s->verts[3 * i + 2]); }

/* splitmix64 (Steele, Lea & Flood 2014) keyed draws in [0, 1). */
static inline uint64_t smix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double u01(uint64_t seed, uint64_t key, uint32_t dim)
{
    return (double)(smix(seed ^ smix(key * 0x100000001B3ull + dim)) >> 11) * (1.0 / 9007199254740992.0);
}

/* Orthonormal frame about n (z axis). */
static void frame(d3 n, d3* x, d3* y)
{
    d3 t = fabs(n.x) > 0.99 ? D3(0, 1, 0) : D3(1, 0, 0);
    *y = dnorm(dcross(n, t));
    *x = dcross(*y, n);
}

/* Malley's method over Shirley-Chiu's concentric disk (core/montecarlo.cu:59-106,153-158). */
static d3 cos_hemi(double u1, double u2)
{
    double sx = 1.0 - 2.0 * u1, sy = 1.0 - 2.0 * u2, r, th;
    if (sx == 0.0 && sy == 0.0) return D3(0, 0, 1);
    if (sx >= -sy) {
        if (sx > sy) { r = sx; th = sy > 0.0 ? sy / r : 8.0 + sy / r; }
        else { r = sy; th = 2.0 - sx / r; }
    } else {
        if (sx <= sy) { r = -sx; th = 4.0 - sy / r; }
        else { r = -sy; th = 6.0 + sx / r; }
    }
    th *= RB2O_PI / 4.0;
    double x = r * cos(th), y = r * sin(th);
    double z = 1.0 - x * x - y * y;
    return D3(x, y, z > 0.0 ? sqrt(z) : 0.0);
}

static inline void mkray(float* r8, d3 o, double tmin, d3 d, double tmax)
{
    r8[0] = (float)o.x; r8[1] = (float)o.y; r8[2] = (float)o.z; r8[3] = (float)tmin;
    r8[4] = (float)d.x; r8[5] = (float)d.y; r8[6] = (float)d.z; r8[7] = (float)tmax;
}

/* Visit counters of the integrator references, per ray type (RB2O_RAY_*):
 * nodes, triangles, leaf terminators, rays; off unless rb2o_counts_reset(1). */
static uint64_t g_cnt[RB2O_RAY_TYPES][4];
static int g_counting = 0;

void rb2o_counts_reset(int on)
{
    memset(g_cnt, 0, sizeof(g_cnt));
    g_counting = on;
}

void rb2o_counts_read(uint64_t* out)
{
    memcpy(out, g_cnt, sizeof(g_cnt));
}

static void trace_ct(const rb2o_bvh* b, const float* r, int any_hit, rb2o_hit* h, int type)
{
    if (!g_counting) {
        trace_one(b->nodes, b->woop, b->triidx, r, any_hit, h, NULL);
        return;
    }
    rb2o_counts c;
    trace_one(b->nodes, b->woop, b->triidx, r, any_hit, h, &c);
#ifdef _OPENMP
#pragma omp atomic
#endif
    g_cnt[type][0] += c.nodes;
#ifdef _OPENMP
#pragma omp atomic
#endif
    g_cnt[type][1] += c.tris;
#ifdef _OPENMP
#pragma omp atomic
#endif
    g_cnt[type][2] += c.leafterms;
#ifdef _OPENMP
#pragma omp atomic
#endif
    g_cnt[type][3] += 1;
}

static inline int occluded_t(const rb2o_bvh* b, const float* r8, int type)
{
    rb2o_hit h;
    trace_ct(b, r8, 1, &h, type);
    return h.prim >= 0;
}
#define occluded(b, r8) occluded_t((b), (r8), RB2O_RAY_SHADOW)

/* The reference's AO direction (core/montecarlo.cu:133-151) about n:
 * returns 0 when its X axis is undefined (n along the axis its signed
 * comparisons pick), where the reference's direction is NaN. */
int rb2o_ao_ref_dir(const double* n3, double u1, double u2, double* out3)
{
    d3 ng = D3(n3[0], n3[1], n3[2]);
    d3 perp = D3(0, 0, 1);
    if (ng.x < ng.y && ng.x < ng.z) perp = D3(1, 0, 0);
    else if (ng.y < ng.x && ng.y < ng.z) perp = D3(0, 1, 0);
    d3 cx = dcross(ng, perp);
    if (!(ddot(cx, cx) > 0.0)) return 0;
    d3 X = dnorm(cx), Y = dnorm(dcross(ng, X));
    double phi = 2.0 * RB2O_PI * u1, theta = acos(sqrt(1.0 - u2));
    d3 w = dadd(dadd(dmul(X, cos(phi) * sin(theta)), dmul(Y, sin(phi) * sin(theta))), dmul(ng, cos(phi)));
    out3[0] = w.x; out3[1] = w.y; out3[2] = w.z;
    return 1;
}

/* DiffuseAreaLight::Le's direction and contribution factor (core/lights.cu:63-69):
 * direction uniform over the hemisphere about world +z (z = u3, phi = 2 pi u4),
 * negated when its dot product with the light normal ln is nonzero; the
 * contribution Le / pdf is Le x k, k = area 2 pi cos for cos = ln . dir > 0,
 * else 0. */
void rb2o_light_le_ref(const double* ln3, double area, double u3, double u4, double* dir3, double* k)
{
    d3 ln = D3(ln3[0], ln3[1], ln3[2]);
    double hr = sqrt(u3 < 1.0 ? 1.0 - u3 * u3 : 0.0), phi = 2.0 * RB2O_PI * u4;
    d3 dir = D3(hr * cos(phi), hr * sin(phi), u3);
    if (ddot(dir, ln) != 0.0) dir = dmul(dir, -1.0);
    double c = ddot(ln, dir);
    dir3[0] = dir.x; dir3[1] = dir.y; dir3[2] = dir.z;
    *k = c > 0.0 ? area * 2.0 * RB2O_PI * c : 0.0;
}

void rb2o_ao(const rb2o_bvh* b, const rb2o_scene* s, const float* prim_rays, uint32_t n, uint32_t samples,
             float radius, uint64_t seed, uint32_t compat, double* out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float* r = prim_rays + 8 * i;
        rb2o_hit h;
        trace_ct(b, r, 0, &h, RB2O_RAY_CAMERA);
        if (h.prim < 0) { out[i] = 0.0; continue; }
        const uint32_t* t = s->tris + 3 * (size_t)h.prim;
        d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
        d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
        d3 d = D3(r[4], r[5], r[6]);
        d3 pos = dadd(D3(r[0], r[1], r[2]), dmul(d, h.t));
        if (compat & 1u) {
            /* The reference's direction formula about the unflipped normal. */
            const double n3[3] = {ng.x, ng.y, ng.z};
            uint64_t open = 0;
            for (uint32_t k = 0; k < samples; k++) {
                uint64_t key = (uint64_t)i * samples + k;
                double w3[3];
                if (!rb2o_ao_ref_dir(n3, u01(seed, key, 0), u01(seed, key, 1), w3)) {
                    open++;  /* the reference's direction is NaN: no hit */
                    continue;
                }
                d3 w = D3(w3[0], w3[1], w3[2]);
                float r8[8];
                mkray(r8, pos, 1.0e-3 * (double)h.t, w, radius);
                if (!occluded(b, r8)) open++;
            }
            out[i] = (double)open / (double)samples;
            continue;
        }
        if (ddot(ng, d) > 0.0) ng = dmul(ng, -1.0);
        d3 fx, fy;
        frame(ng, &fx, &fy);
        uint64_t open = 0;
        for (uint32_t k = 0; k < samples; k++) {
            uint64_t key = (uint64_t)i * samples + k;
            d3 l = cos_hemi(u01(seed, key, 0), u01(seed, key, 1));
            d3 w = dadd(dadd(dmul(fx, l.x), dmul(fy, l.y)), dmul(ng, l.z));
            float r8[8];
            mkray(r8, pos, 1.0e-3 * (double)h.t, w, radius);
            if (!occluded(b, r8)) open++;
        }
        out[i] = (double)open / (double)samples;
    }
    (void)nthreads;
}

static double tri_area_d(d3 a, d3 b_, d3 c)
{
    d3 cr = dcross(dsub(b_, a), dsub(c, a));
    return 0.5 * sqrt(ddot(cr, cr));
}

/* ---- layered materials (FP64) ---------------------------------------------------- */
typedef struct { d3 x, y, z; } frame3;
static frame3 frame_z(d3 n)
{
    frame3 f;
    f.z = dnorm(n);
    d3 t = fabs(f.z.x) > 0.99 ? D3(0, 1, 0) : D3(1, 0, 0);
    f.y = dnorm(dcross(f.z, t));
    f.x = dcross(f.y, f.z);
    return f;
}
static d3 fr_local(const frame3* f, d3 w) { return D3(ddot(w, f->x), ddot(w, f->y), ddot(w, f->z)); }
static d3 fr_world(const frame3* f, d3 w) { return dadd(dadd(dmul(f->x, w.x), dmul(f->y, w.y)), dmul(f->z, w.z)); }
static int same_h(d3 a, d3 b) { return a.z * b.z > 0.0; }
static double sin2t(d3 w) { double v = 1.0 - w.z * w.z; return v > 0.0 ? v : 0.0; }
static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int is_delta(uint32_t k) { return k == 2 || k == 3; }
static uint32_t bx_bits(uint32_t k) { return k == 2 ? (1u | 16u) : (k == 3 ? (1u | 16u | 2u) : (k == 4 ? (1u | 8u) : (1u | 4u))); }

static double fres_diel(double cosi, double etai, double etat)
{
    int entering = cosi > 0.0;
    double ei = entering ? etai : etat, et = entering ? etat : etai;
    double sint = ei / et * sqrt(1.0 - cosi * cosi > 0.0 ? 1.0 - cosi * cosi : 0.0);
    if (sint >= 1.0) return 1.0;
    double cost = sqrt(1.0 - sint * sint > 0.0 ? 1.0 - sint * sint : 0.0), ci = fabs(cosi);
    double rpar = (et * ci - ei * cost) / (et * ci + ei * cost);
    double rperp = (ei * ci - et * cost) / (ei * ci + et * cost);
    return (rpar * rpar + rperp * rperp) / 2.0;
}
static double fres_cond(double cosi, double eta, double k)
{
    double tmp = (eta * eta + k * k) * cosi * cosi;
    double rpar2 = (tmp - 2.0 * eta * cosi + 1.0) / (tmp + 2.0 * eta * cosi + 1.0);
    double tf = eta * eta + k * k;
    double rperp2 = (tf - 2.0 * eta * cosi + cosi * cosi) / (tf + 2.0 * eta * cosi + cosi * cosi);
    return (rpar2 + rperp2) / 2.0;
}
static d3 fres(const rb2o_layer* l, double cosi)
{
    if (l->fresnel == 1) return D3(fres_cond(cosi, l->eta[0], l->k[0]), fres_cond(cosi, l->eta[1], l->k[1]),
                                   fres_cond(cosi, l->eta[2], l->k[2]));
    if (l->fresnel == 0) { double r = fres_diel(clampd(cosi, -1.0, 1.0), l->etai, l->etat); return D3(r, r, r); }
    return D3(1, 1, 1);
}
static d3 col(const rb2o_layer* l) { return D3(l->color[0], l->color[1], l->color[2]); }
static double blinn_D_d(d3 wh, double e) { return (e + 2.0) / (2.0 * RB2O_PI) * pow(fabs(wh.z), e); }
static double blinn_pdf_d(d3 wo, d3 wi, double e)
{
    d3 wh = dnorm(dadd(wo, wi));
    double d = ddot(wo, wh);
    if (d <= 0.0) return 0.0;
    return ((e + 1.0) * pow(fabs(wh.z), e)) / (2.0 * RB2O_PI * 4.0 * d);
}
static d3 mf_eval(const rb2o_layer* l, d3 wi, d3 wo)
{
    double co = fabs(wo.z), ci = fabs(wi.z);
    if (ci == 0.0 || co == 0.0) return D3(0, 0, 0);
    d3 wh = dadd(wi, wo);
    if (wh.x == 0.0 && wh.y == 0.0 && wh.z == 0.0) return D3(0, 0, 0);
    wh = dnorm(wh);
    d3 F = fres(l, ddot(wi, wh));
    double nh = fabs(wh.z), woh = fabs(ddot(wo, wh));
    double g1 = 2.0 * nh / woh, g2 = 2.0 * nh * ci / woh;
    double G = 1.0;
    if (g1 < G) G = g1;
    if (g2 < G) G = g2;
    double s = blinn_D_d(wh, l->exponent) * G / (4.0 * ci * co);
    return D3(l->color[0] * s * F.x, l->color[1] * s * F.y, l->color[2] * s * F.z);
}
static void on_AB(const rb2o_layer* l, double* A, double* B)
{
    double sd = l->sigma_deg < 0.0f ? 0.0 : (l->sigma_deg > 90.0f ? 90.0 : (double)l->sigma_deg);
    double sg = sd * RB2O_PI / 180.0, s2 = sg * sg;
    *A = 1.0 - s2 / (2.0 * (s2 + 0.33));
    *B = 0.45 * s2 / (s2 + 0.09);
}
static d3 on_eval(const rb2o_layer* l, d3 wi, d3 wo)
{
    double si = sqrt(sin2t(wi)), so = sqrt(sin2t(wo)), maxcos = 0.0;
    if (si > 1e-4 && so > 1e-4) {
        double cpi = si == 0.0 ? 1.0 : clampd(wi.x / si, -1, 1), spi = si == 0.0 ? 0.0 : clampd(wi.y / si, -1, 1);
        double cpo = so == 0.0 ? 1.0 : clampd(wo.x / so, -1, 1), spo = so == 0.0 ? 0.0 : clampd(wo.y / so, -1, 1);
        double dc = cpi * cpo + spi * spo;
        maxcos = dc > 0.0 ? dc : 0.0;
    }
    double sa, tb;
    if (fabs(wi.z) > fabs(wo.z)) { sa = so; tb = si / fabs(wi.z); }
    else { sa = si; tb = so / fabs(wo.z); }
    double A, B;
    on_AB(l, &A, &B);
    return dmul(col(l), (A + B * maxcos * sa * tb) / RB2O_PI);
}
static d3 layer_f_d(const rb2o_layer* l, d3 wi, d3 wo)
{
    switch (l->type) {
    case 0: return same_h(wi, wo) ? dmul(col(l), 1.0 / RB2O_PI) : D3(0, 0, 0);
    case 1: return on_eval(l, wi, wo);
    case 4: return mf_eval(l, wi, wo);
    default: return D3(0, 0, 0);
    }
}
static double layer_pdf_d(const rb2o_layer* l, d3 wi, d3 wo)
{
    if (l->type == 0 || l->type == 1) return same_h(wi, wo) ? fabs(wi.z) / RB2O_PI : 0.0;
    if (l->type == 4) return same_h(wi, wo) ? blinn_pdf_d(wo, wi, l->exponent) : 0.0;
    return 0.0;
}
static d3 mat_f(const rb2o_material* m, d3 n, d3 wo_w, d3 wi_w, d3 wo, d3 wi)
{
    uint32_t side = ddot(wi_w, n) * ddot(wo_w, n) > 0.0 ? (1u | 4u | 8u) : (2u | 4u | 8u);
    d3 f = D3(0, 0, 0);
    for (uint32_t i = 0; i < m->n_layers; i++) {
        uint32_t bits = bx_bits(m->layer[i].type);
        if ((bits & side) != bits) continue;
        f = dadd(f, layer_f_d(&m->layer[i], wi, wo));
    }
    return f;
}
static double mat_pdf(const rb2o_material* m, d3 wo, d3 wi)
{
    double p = 0.0;
    uint32_t n = 0;
    for (uint32_t i = 0; i < m->n_layers; i++) {
        if (is_delta(m->layer[i].type)) continue;
        n++;
        p += layer_pdf_d(&m->layer[i], wi, wo);
    }
    return n ? p / n : 0.0;
}
/* Returns f; wi_w, pdf, specular out. */
/* eta_io (nullable): for a sampled glass layer, the index of wo's side over
 * wi's side (1 otherwise). */
static d3 mat_sample(const rb2o_material* m, d3 n, d3 wo_w, double u1, double u2, double uc, d3* wi_w, double* pdf,
                     int* specular, double* eta_io)
{
    *pdf = 0.0;
    *specular = 0;
    if (eta_io) *eta_io = 1.0;
    if (m->n_layers == 0) return D3(0, 0, 0);
    frame3 fr = frame_z(n);
    d3 wo = fr_local(&fr, wo_w);
    uint32_t which = (uint32_t)floor(uc * m->n_layers);
    if (which > m->n_layers - 1) which = m->n_layers - 1;
    const rb2o_layer* l = &m->layer[which];
    d3 wi, f;
    if (l->type == 2) {
        wi = D3(-wo.x, -wo.y, wo.z);
        *pdf = 1.0;
        f = dmul(col(l), 1.0 / fabs(wi.z));
    } else if (l->type == 3) {
        int entering = wo.z > 0.0;
        double ei = entering ? l->etai : l->etat, et = entering ? l->etat : l->etai, eta = ei / et;
        double sint2 = eta * eta * sin2t(wo);
        if (sint2 >= 1.0) return D3(0, 0, 0);
        double cost = sqrt(1.0 - sint2 > 0.0 ? 1.0 - sint2 : 0.0);
        if (entering) cost = -cost;
        wi = D3(eta * -wo.x, eta * -wo.y, cost);
        *pdf = 1.0;
        double F = fres_diel(wo.z, l->etai, l->etat);
        f = dmul(col(l), (et * et) / (ei * ei) * (1.0 - F) / fabs(wi.z));
        if (eta_io) *eta_io = ei / et;
    } else if (l->type == 4) {
        double e = l->exponent, ct = pow(u1, 1.0 / (e + 1.0)), st = sqrt(1.0 - ct * ct > 0.0 ? 1.0 - ct * ct : 0.0);
        double phi = u2 * 2.0 * RB2O_PI;
        d3 wh = D3(st * cos(phi), st * sin(phi), ct);
        if (!same_h(wo, wh)) wh = dmul(wh, -1.0);
        double d = ddot(wo, wh);
        wi = dadd(dmul(wo, -1.0), dmul(wh, 2.0 * d));
        *pdf = d <= 0.0 ? 0.0 : ((e + 1.0) * pow(ct, e)) / (2.0 * RB2O_PI * 4.0 * d);
        f = same_h(wi, wo) ? mf_eval(l, wi, wo) : D3(0, 0, 0);
    } else {
        wi = cos_hemi(u1, u2);
        if (wo.z < 0.0) wi.z = -wi.z;
        wi = dnorm(wi);
        *pdf = same_h(wi, wo) ? fabs(wi.z) / RB2O_PI : 0.0;
        f = layer_f_d(l, wi, wo);
    }
    if (*pdf == 0.0) return D3(0, 0, 0);
    *wi_w = fr_world(&fr, wi);
    *specular = is_delta(l->type);
    if (!*specular) {
        for (uint32_t i = 0; i < m->n_layers; i++)
            if (i != which && !is_delta(m->layer[i].type)) *pdf += layer_pdf_d(&m->layer[i], wi, wo);
        f = mat_f(m, n, wo_w, *wi_w, wo, wi);
    }
    *pdf /= m->n_layers;
    return f;
}

void rb2o_material_query(const rb2o_material* m, int sample, const double* q, double* out)
{
    d3 n = D3(q[0], q[1], q[2]), wo_w = D3(q[3], q[4], q[5]);
    if (sample) {
        d3 wi = D3(0, 0, 0);
        double pdf;
        int spec;
        d3 f = mat_sample(m, n, wo_w, q[6], q[7], q[8], &wi, &pdf, &spec, NULL);
        out[0] = wi.x; out[1] = wi.y; out[2] = wi.z; out[3] = f.x; out[4] = f.y; out[5] = f.z; out[6] = pdf;
        out[7] = spec;
    } else {
        frame3 fr = frame_z(n);
        d3 wi_w = D3(q[6], q[7], q[8]);
        d3 wo = fr_local(&fr, wo_w), wi = fr_local(&fr, wi_w);
        d3 f = mat_f(m, n, wo_w, wi_w, wo, wi);
        out[0] = f.x; out[1] = f.y; out[2] = f.z; out[3] = mat_pdf(m, wo, wi);
    }
}

static int plain_lambertian(const rb2o_material* m) { return m->n_layers == 1 && m->layer[0].type == 0; }
static int has_nondelta(const rb2o_material* m)
{
    for (uint32_t i = 0; i < m->n_layers; i++)
        if (!is_delta(m->layer[i].type)) return 1;
    return 0;
}

/* Russian roulette after the BSDF sample at bounce bnc: from bounce rr_start
 * dividing survivors by q, or (compat bit 2) from rr_start + 1 dividing by
 * 1 - q (integrator_path.cu:232-244).  Returns 0 when the path ends. */
static int rr_step(double* T, uint32_t bnc, uint32_t rr_start, float rr_prob, uint32_t compat, double u)
{
    const int ref = (compat & 2u) != 0;
    if (ref ? bnc <= rr_start : bnc < rr_start) return 1;
    double lum = 0.212671 * T[0] + 0.715160 * T[1] + 0.072169 * T[2];
    double q = lum < rr_prob ? lum : rr_prob;
    if (!(u < q)) return 0;
    double div = ref ? 1.0 - q : q;
    for (int c = 0; c < 3; c++) T[c] /= div;
    return 1;
}

void rb2o_pt(const rb2o_bvh* b, const rb2o_scene* s, const float* rays, uint32_t n, uint32_t max_depth,
             uint32_t rr_start, float rr_prob, uint64_t seed, uint32_t compat, double* out_rgb, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        double L[3] = {0, 0, 0}, T[3] = {1, 1, 1}, pdf_prev = 0.0;
        float ray[8];
        for (int k = 0; k < 8; k++) ray[k] = rays[8 * i + k];
        const double inv_nl = s->n_lights ? 1.0 / (double)s->n_lights : 0.0;
        for (uint32_t bnc = 0;; bnc++) {
            rb2o_hit h;
            trace_ct(b, ray, 0, &h, bnc == 0 ? RB2O_RAY_CAMERA : RB2O_RAY_EXTENSION);
            if (h.prim < 0) break;
            const uint32_t* t = s->tris + 3 * (size_t)h.prim;
            const uint32_t m = s->tri_mat[h.prim];
            d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
            d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
            d3 d = D3(ray[4], ray[5], ray[6]);
            d3 wo = dmul(d, -1.0);
            d3 pos = dadd(D3(ray[0], ray[1], ray[2]), dmul(d, h.t));
            const double eps = 1.0e-3 * (double)h.t;
            const float* E = s->emission + 3 * (size_t)m;
            if (E[0] > 0.0f || E[1] > 0.0f || E[2] > 0.0f) {
                double cosl = ddot(ng, wo);
                if (cosl > 0.0) {
                    double w = 1.0;
                    if (bnc > 0 && pdf_prev > 0.0) {  /* pdf_prev < 0: specular bounce */
                        double pdf_l = inv_nl * (double)h.t * (double)h.t / (tri_area_d(v0, v1, v2) * cosl);
                        w = pdf_prev / (pdf_prev + pdf_l);
                    }
                    for (int c = 0; c < 3; c++) L[c] += T[c] * E[c] * w;
                }
                break;
            }
            uint64_t key = (uint64_t)i * 64 + bnc;
            /* NEE draws: this vertex's, or (compat bit 4) the first vertex's at every
             * vertex, as the reference re-seeds its NEE generator (integrator_path.cu:113). */
            uint64_t nkey = (compat & 4u) ? (uint64_t)i * 64 : key;
            if (s->materials && !plain_lambertian(&s->materials[m])) {
                /* Layered material: NEE with material_f / material_pdf (skipped for
                 * purely specular materials), continuation by material_sample_f;
                 * emission after a specular bounce takes full weight. */
                const rb2o_material* mt = &s->materials[m];
                frame3 fr = frame_z(ng);
                d3 wo_l = fr_local(&fr, wo);
                if (s->n_lights && has_nondelta(mt)) {
                    uint32_t j = (uint32_t)(u01(seed, nkey, 0) * s->n_lights);
                    if (j >= s->n_lights) j = s->n_lights - 1;
                    const uint32_t lt = s->lights[j];
                    const uint32_t* lv = s->tris + 3 * (size_t)lt;
                    d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
                    double su = sqrt(u01(seed, nkey, 1)), u2 = u01(seed, nkey, 2);
                    double b0 = 1.0 - su, b1 = u2 * su;
                    d3 lp = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
                    d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
                    d3 dv = dsub(lp, pos);
                    double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                    d3 wi = dmul(dv, 1.0 / dist);
                    double cos_l = -ddot(ln, wi);
                    const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
                    if (cos_l > 0.0 && dist > 0.0) {
                        d3 wi_l = fr_local(&fr, wi);
                        d3 f = mat_f(mt, ng, wo, wi, wo_l, wi_l);
                        if (f.x > 0.0 || f.y > 0.0 || f.z > 0.0) {
                            double pdf_l = inv_nl * dist2 / (tri_area_d(l0, l1, l2) * cos_l);
                            double pdf_b = mat_pdf(mt, wo_l, wi_l);
                            double w = (bnc == max_depth) ? 1.0 : pdf_l / (pdf_l + pdf_b);
                            float sr[8];
                            mkray(sr, pos, eps, wi, dist * (1.0 - 1.0e-3));
                            if (!occluded(b, sr)) {
                                double k = fabs(ddot(wi, ng)) * w / pdf_l;
                                L[0] += T[0] * f.x * Le[0] * k;
                                L[1] += T[1] * f.y * Le[1] * k;
                                L[2] += T[2] * f.z * Le[2] * k;
                            }
                        }
                    }
                }
                if (bnc >= max_depth) break;
                d3 wi = D3(0, 0, 0);
                double pdf;
                int spec;
                d3 f = mat_sample(mt, ng, wo, u01(seed, key, 3), u01(seed, key, 4), u01(seed, key, 6), &wi, &pdf, &spec,
                                  NULL);
                if (!(pdf > 0.0) || !(f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) break;
                double k = fabs(ddot(wi, ng)) / pdf;
                T[0] *= f.x * k; T[1] *= f.y * k; T[2] *= f.z * k;
                pdf_prev = spec ? -1.0 : pdf;
                if (!rr_step(T, bnc, rr_start, rr_prob, compat, u01(seed, key, 5))) break;
                mkray(ray, pos, eps, wi, 3.402823466e+38);
                continue;
            }
            d3 nrm = ddot(ng, wo) < 0.0 ? dmul(ng, -1.0) : ng;
            const float* A = s->albedo + 3 * (size_t)m;
            if (s->n_lights) {
                uint32_t j = (uint32_t)(u01(seed, nkey, 0) * s->n_lights);
                if (j >= s->n_lights) j = s->n_lights - 1;
                const uint32_t lt = s->lights[j];
                const uint32_t* lv = s->tris + 3 * (size_t)lt;
                d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
                double su = sqrt(u01(seed, nkey, 1)), u2 = u01(seed, nkey, 2);
                double b0 = 1.0 - su, b1 = u2 * su;
                d3 lp = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
                d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
                d3 dv = dsub(lp, pos);
                double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                d3 wi = dmul(dv, 1.0 / dist);
                double cos_l = -ddot(ln, wi), cos_s = ddot(nrm, wi);
                const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
                if (cos_l > 0.0 && cos_s > 0.0 && dist > 0.0) {
                    double pdf_l = inv_nl * dist2 / (tri_area_d(l0, l1, l2) * cos_l);
                    double pdf_b = cos_s / RB2O_PI;
                    double w = (bnc == max_depth) ? 1.0 : pdf_l / (pdf_l + pdf_b);
                    float sr[8];
                    mkray(sr, pos, eps, wi, dist * (1.0 - 1.0e-3));
                    if (!occluded(b, sr))
                        for (int c = 0; c < 3; c++) L[c] += T[c] * (A[c] / RB2O_PI) * Le[c] * cos_s * w / pdf_l;
                }
            }
            if (bnc >= max_depth) break;
            d3 fx, fy;
            frame(nrm, &fx, &fy);
            d3 l = cos_hemi(u01(seed, key, 3), u01(seed, key, 4));
            double pdf = l.z / RB2O_PI;
            if (!(pdf > 0.0)) break;
            d3 wi = dnorm(dadd(dadd(dmul(fx, l.x), dmul(fy, l.y)), dmul(nrm, l.z)));
            for (int c = 0; c < 3; c++) T[c] *= A[c];
            pdf_prev = pdf;
            if (T[0] <= 0.0 && T[1] <= 0.0 && T[2] <= 0.0) break;
            if (!rr_step(T, bnc, rr_start, rr_prob, compat, u01(seed, key, 5))) break;
            mkray(ray, pos, eps, wi, 3.402823466e+38);
        }
        for (int c = 0; c < 3; c++) out_rgb[3 * i + c] = L[c];
    }
    (void)nthreads;
}

/* ---- BDPT with a light-vertex cache ------------------------------------------------
 * Per iteration: n_light_paths light subpaths (uniform emissive triangle,
 * uniform point, cosine direction), every non-emitter surface vertex y1..y_Dl
 * cached (Dl = K - 2); then one camera path per camera ray with emission
 * (s = 0), NEE (s = 1) and C uniform cache connections (s >= 2, scaled by
 * cache size / light paths).  A k-segment path is sampled by emission and by a
 * connection across each edge whose endpoints both scatter non-specularly (the
 * camera counts as specular, the light point not); each of those n strategies
 * is weighted 1/n (1/k without specular vertices).  Vertices of purely
 * specular materials are not cached. */
/* el: valid connection edges on the light side with this vertex as a
 * (non-specular) endpoint; see the strategy counting in rb2o_bdpt. */
typedef struct { d3 pos, nrm, beta, wi, ng; double el; uint32_t s, mat; } lvc_vertex;

void rb2o_bdpt(const rb2o_bvh* b, const rb2o_scene* s, const float* cam_rays, uint32_t n_cam, uint32_t n_iter,
               uint32_t n_light_paths, uint32_t K, uint32_t C, uint32_t rr_start, float rr_prob, uint64_t seed,
               double* out_rgb, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    const uint32_t Dl = K >= 2 ? K - 2 : 0;
    const double inv_nl = s->n_lights ? 1.0 / (double)s->n_lights : 0.0;
    lvc_vertex* sparse = (lvc_vertex*)calloc((size_t)n_light_paths * (Dl ? Dl : 1), sizeof(lvc_vertex));
    uint8_t* valid = (uint8_t*)calloc((size_t)n_light_paths * (Dl ? Dl : 1), 1);
    lvc_vertex* dense = (lvc_vertex*)calloc((size_t)n_light_paths * (Dl ? Dl : 1), sizeof(lvc_vertex));
    for (size_t i = 0; i < (size_t)n_cam * 3; i++) out_rgb[i] = 0.0;
    for (uint32_t it = 0; it < n_iter; it++) {
        memset(valid, 0, (size_t)n_light_paths * (Dl ? Dl : 1));
        const uint64_t ls = seed ^ 0xA24BAED4963EE407ull;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
        for (int64_t p = 0; p < (int64_t)n_light_paths; p++) {
            if (!s->n_lights || Dl == 0) continue;
            const uint64_t key = (uint64_t)it * n_light_paths + (uint64_t)p;
            uint32_t j = (uint32_t)(u01(ls, key, 0) * s->n_lights);
            if (j >= s->n_lights) j = s->n_lights - 1;
            const uint32_t lt = s->lights[j];
            const uint32_t* lv = s->tris + 3 * (size_t)lt;
            d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
            double su = sqrt(u01(ls, key, 1)), u2 = u01(ls, key, 2);
            double b0 = 1.0 - su, b1 = u2 * su;
            d3 y0 = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
            d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
            d3 fx, fy;
            frame(ln, &fx, &fy);
            d3 l = cos_hemi(u01(ls, key, 3), u01(ls, key, 4));
            d3 dir = dnorm(dadd(dadd(dmul(fx, l.x), dmul(fy, l.y)), dmul(ln, l.z)));
            const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
            double kk = (double)s->n_lights * tri_area_d(l0, l1, l2) * RB2O_PI;
            double beta[3] = {Le[0] * kk, Le[1] * kk, Le[2] * kk};
            float ray[8];
            mkray(ray, y0, 1.0e-4, dir, 3.402823466e+38);
            int nsp_prev = 1;      /* the light point scatters non-specularly */
            uint32_t edges = 0;    /* valid connection edges so far */
            for (uint32_t d = 1; d <= Dl; d++) {
                rb2o_hit h;
                trace_ct(b, ray, 0, &h, RB2O_RAY_LIGHT);
                if (h.prim < 0) break;
                const uint32_t* t = s->tris + 3 * (size_t)h.prim;
                const uint32_t m = s->tri_mat[h.prim];
                const float* E = s->emission + 3 * (size_t)m;
                if (E[0] > 0.0f || E[1] > 0.0f || E[2] > 0.0f) break;
                d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
                d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
                d3 dd = D3(ray[4], ray[5], ray[6]);
                d3 wo = dmul(dd, -1.0);
                d3 nrm = ddot(ng, wo) < 0.0 ? dmul(ng, -1.0) : ng;
                d3 pos = dadd(D3(ray[0], ray[1], ray[2]), dmul(dd, h.t));
                size_t slot = (size_t)p * Dl + (d - 1);
                /* Purely specular vertices cannot be connected to: not cached. */
                if (!s->materials || plain_lambertian(&s->materials[m]) || has_nondelta(&s->materials[m])) {
                    sparse[slot].pos = pos; sparse[slot].nrm = nrm;
                    sparse[slot].beta = D3(beta[0], beta[1], beta[2]);
                    sparse[slot].s = d + 1; sparse[slot].mat = m;
                    sparse[slot].wi = wo; sparse[slot].ng = ng;
                    sparse[slot].el = (double)(edges + (uint32_t)nsp_prev);
                    valid[slot] = 1;
                }
                if (d >= Dl) break;
                if (s->materials && !plain_lambertian(&s->materials[m])) {
                    /* Layered (non-specular) material: sample its BSDF toward the next light vertex. */
                    d3 wn = D3(0, 0, 0);
                    double pdf, eta_io;
                    int spec;
                    d3 f = mat_sample(&s->materials[m], ng, wo, u01(ls, key, 8 + 8 * d), u01(ls, key, 9 + 8 * d),
                                      u01(ls, key, 11 + 8 * d), &wn, &pdf, &spec, &eta_io);
                    if (!(pdf > 0.0) || !(f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) break;
                    if (!spec) {
                        /* Light flows from wo toward wn: the adjoint f(wn -> wo) (the Blinn
                         * shadowing term is not symmetric in its two directions). */
                        frame3 frl = frame_z(ng);
                        f = mat_f(&s->materials[m], ng, wn, wo, fr_local(&frl, wn), fr_local(&frl, wo));
                    } else {
                        /* Adjoint of a glass transmission: (eta_o / eta_i)^6 times the
                         * sampled factor (the camera-side (eta_i / eta_o)^2 and the solid
                         * angle map of the refraction); 1 for a mirror. */
                        double e2 = eta_io * eta_io;
                        f = dmul(f, e2 * e2 * e2);
                    }
                    double k = fabs(ddot(wn, nrm)) / pdf;
                    double fac[3] = {f.x * k, f.y * k, f.z * k};
                    double lum = 0.212671 * fac[0] + 0.715160 * fac[1] + 0.072169 * fac[2];
                    double q = lum < 1.0 ? lum : 1.0;
                    if (d < rr_start) q = 1.0; else if (q > rr_prob) q = rr_prob;
                    if (!(q > 0.0 && u01(ls, key, 10 + 8 * d) < q)) break;
                    for (int c2 = 0; c2 < 3; c2++) beta[c2] *= fac[c2] / q;
                    edges += (nsp_prev && !spec) ? 1u : 0u;
                    nsp_prev = !spec;
                    mkray(ray, pos, 1.0e-3 * (double)h.t, wn, 3.402823466e+38);
                    continue;
                }
                const float* A = s->albedo + 3 * (size_t)m;
                d3 lc = cos_hemi(u01(ls, key, 8 + 8 * d), u01(ls, key, 9 + 8 * d));
                if (!(lc.z > 0.0)) break;
                frame(nrm, &fx, &fy);
                d3 wi = dnorm(dadd(dadd(dmul(fx, lc.x), dmul(fy, lc.y)), dmul(nrm, lc.z)));
                double lum = 0.212671 * A[0] + 0.715160 * A[1] + 0.072169 * A[2];
                double q = lum < 1.0 ? lum : 1.0;
                if (d < rr_start) q = 1.0; else if (q > rr_prob) q = rr_prob;
                if (!(q > 0.0 && u01(ls, key, 10 + 8 * d) < q)) break;
                for (int c = 0; c < 3; c++) beta[c] *= A[c] / q;
                edges += nsp_prev ? 1u : 0u;
                nsp_prev = 1;
                mkray(ray, pos, 1.0e-3 * (double)h.t, wi, 3.402823466e+38);
            }
        }
        uint32_t M = 0;
        for (size_t i = 0; i < (size_t)n_light_paths * Dl; i++)
            if (valid[i]) dense[M++] = sparse[i];
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
        for (int64_t ci = 0; ci < (int64_t)n_cam; ci++) {
            double L[3] = {0, 0, 0}, T[3] = {1, 1, 1};
            /* Strategy counting: a k-segment path is weighted 1 / n_valid, n_valid =
             * 1 + (edges whose endpoints both scatter non-specularly); cnsp: the
             * previous camera vertex scattered non-specularly (the camera counts as
             * specular), cedges: valid edges among the camera vertices so far. */
            int cnsp = 0;
            uint32_t cedges = 0;
            float ray[8];
            for (int k = 0; k < 8; k++) ray[k] = cam_rays[8 * ((size_t)it * n_cam + ci) + k];
            const uint64_t key = (uint64_t)it * n_cam + (uint64_t)ci;
            for (uint32_t i = 1; i <= K; i++) {
                rb2o_hit h;
                trace_ct(b, ray, 0, &h, i == 1 ? RB2O_RAY_CAMERA : RB2O_RAY_EXTENSION);
                if (h.prim < 0) break;
                const uint32_t* t = s->tris + 3 * (size_t)h.prim;
                const uint32_t m = s->tri_mat[h.prim];
                d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
                d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
                d3 dd = D3(ray[4], ray[5], ray[6]);
                d3 wo = dmul(dd, -1.0);
                d3 pos = dadd(D3(ray[0], ray[1], ray[2]), dmul(dd, h.t));
                const double eps = 1.0e-3 * (double)h.t;
                const float* E = s->emission + 3 * (size_t)m;
                if (E[0] > 0.0f || E[1] > 0.0f || E[2] > 0.0f) {
                    if (ddot(ng, wo) > 0.0)
                        for (int c = 0; c < 3; c++) L[c] += T[c] * E[c] / (double)(1u + cedges + (uint32_t)cnsp);
                    break;
                }
                d3 nrm = ddot(ng, wo) < 0.0 ? dmul(ng, -1.0) : ng;
                const float* A = s->albedo + 3 * (size_t)m;
                uint64_t vkey = key * 64 + i;
                /* Layered materials (non-specular): f from the material functions,
                 * in the frame of the geometric normal as the path tracer uses. */
                const rb2o_material* mc = (s->materials && !plain_lambertian(&s->materials[m])) ? &s->materials[m] : NULL;
                frame3 frc = frame_z(ng);
                d3 wo_l = fr_local(&frc, wo);
                if (s->n_lights && i + 1 <= K) {
                    uint32_t j = (uint32_t)(u01(seed, vkey, 0) * s->n_lights);
                    if (j >= s->n_lights) j = s->n_lights - 1;
                    const uint32_t lt = s->lights[j];
                    const uint32_t* lv = s->tris + 3 * (size_t)lt;
                    d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
                    double su = sqrt(u01(seed, vkey, 1)), u2 = u01(seed, vkey, 2);
                    double b0 = 1.0 - su, b1 = u2 * su;
                    d3 lp = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
                    d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
                    d3 dv = dsub(lp, pos);
                    double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                    d3 wi = dmul(dv, 1.0 / dist);
                    double cos_l = -ddot(ln, wi), cos_s = ddot(nrm, wi);
                    const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
                    if (mc && cos_l > 0.0 && dist > 0.0) {
                        d3 f = mat_f(mc, ng, wo, wi, wo_l, fr_local(&frc, wi));
                        if (f.x > 0.0 || f.y > 0.0 || f.z > 0.0) {
                            double pdf_l = inv_nl * dist2 / (tri_area_d(l0, l1, l2) * cos_l);
                            float sr[8];
                            mkray(sr, pos, eps, wi, dist * (1.0 - 1.0e-3));
                            if (!occluded(b, sr)) {
                                double k = fabs(cos_s) / pdf_l / (double)(2u + cedges + (uint32_t)cnsp);
                                L[0] += T[0] * f.x * Le[0] * k;
                                L[1] += T[1] * f.y * Le[1] * k;
                                L[2] += T[2] * f.z * Le[2] * k;
                            }
                        }
                    } else if (!mc && cos_l > 0.0 && cos_s > 0.0 && dist > 0.0) {
                        double pdf_l = inv_nl * dist2 / (tri_area_d(l0, l1, l2) * cos_l);
                        float sr[8];
                        mkray(sr, pos, eps, wi, dist * (1.0 - 1.0e-3));
                        if (!occluded(b, sr))
                            for (int c = 0; c < 3; c++)
                                L[c] += T[c] * (A[c] / RB2O_PI) * Le[c] * cos_s / pdf_l /
                                        (double)(2u + cedges + (uint32_t)cnsp);
                    }
                }
                if (M > 0 && i + 2 <= K) {
                    for (uint32_t cidx = 0; cidx < C; cidx++) {
                        uint32_t v = (uint32_t)(u01(seed, vkey, 16 + cidx) * M);
                        if (v >= M) v = M - 1;
                        const lvc_vertex* V = &dense[v];
                        if (V->s + i > K) continue;
                        d3 dv = dsub(V->pos, pos);
                        double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                        if (!(dist > 0.0)) continue;
                        d3 dir = dmul(dv, 1.0 / dist);
                        double cos_c = ddot(nrm, dir), cos_v = -ddot(V->nrm, dir);
                        const rb2o_material* mv =
                            (s->materials && !plain_lambertian(&s->materials[V->mat])) ? &s->materials[V->mat] : NULL;
                        if (mc || mv) {
                            /* f at both ends from the material functions (Lambertian: A / pi on the lit side). */
                            d3 fc = mc ? mat_f(mc, ng, wo, dir, wo_l, fr_local(&frc, dir))
                                       : (cos_c > 0.0 ? dmul(D3(A[0], A[1], A[2]), 1.0 / RB2O_PI) : D3(0, 0, 0));
                            d3 fv;
                            if (mv) {
                                frame3 frv = frame_z(V->ng);
                                d3 wov = dmul(dir, -1.0);
                                fv = mat_f(mv, V->ng, wov, V->wi, fr_local(&frv, wov), fr_local(&frv, V->wi));
                            } else {
                                const float* Av = s->albedo + 3 * (size_t)V->mat;
                                fv = cos_v > 0.0 ? dmul(D3(Av[0], Av[1], Av[2]), 1.0 / RB2O_PI) : D3(0, 0, 0);
                            }
                            d3 ff = D3(fc.x * fv.x, fc.y * fv.y, fc.z * fv.z);
                            if (!(ff.x > 0.0 || ff.y > 0.0 || ff.z > 0.0)) continue;
                            float cr[8];
                            mkray(cr, pos, eps, dir, dist * (1.0 - 1.0e-3));
                            if (occluded_t(b, cr, RB2O_RAY_CONNECTION)) continue;
                            double g = fabs(cos_c) * fabs(cos_v) / dist2 * ((double)M / (double)n_light_paths) /
                                       ((2.0 + (double)cedges + (double)cnsp + V->el) * (double)C);
                            L[0] += T[0] * ff.x * V->beta.x * g;
                            L[1] += T[1] * ff.y * V->beta.y * g;
                            L[2] += T[2] * ff.z * V->beta.z * g;
                            continue;
                        }
                        if (!(cos_c > 0.0 && cos_v > 0.0)) continue;
                        float cr[8];
                        mkray(cr, pos, eps, dir, dist * (1.0 - 1.0e-3));
                        if (occluded_t(b, cr, RB2O_RAY_CONNECTION)) continue;
                        const float* Av = s->albedo + 3 * (size_t)V->mat;
                        double g = cos_c * cos_v / dist2 / (RB2O_PI * RB2O_PI) * ((double)M / (double)n_light_paths) /
                                   ((2.0 + (double)cedges + (double)cnsp + V->el) * (double)C);
                        double bv[3] = {V->beta.x, V->beta.y, V->beta.z};
                        for (int c = 0; c < 3; c++) L[c] += T[c] * A[c] * Av[c] * bv[c] * g;
                    }
                }
                if (i >= K) break;
                if (mc) {
                    d3 wn = D3(0, 0, 0);
                    double pdf;
                    int spec;
                    d3 f = mat_sample(mc, ng, wo, u01(seed, vkey, 3), u01(seed, vkey, 4), u01(seed, vkey, 6), &wn, &pdf,
                                      &spec, NULL);
                    if (!(pdf > 0.0) || !(f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) break;
                    double k = fabs(ddot(wn, nrm)) / pdf;
                    T[0] *= f.x * k; T[1] *= f.y * k; T[2] *= f.z * k;
                    if (i - 1 >= rr_start) {
                        double lum = 0.212671 * T[0] + 0.715160 * T[1] + 0.072169 * T[2];
                        double q = lum < rr_prob ? lum : rr_prob;
                        if (!(u01(seed, vkey, 5) < q)) break;
                        for (int c = 0; c < 3; c++) T[c] /= q;
                    }
                    cedges += (cnsp && !spec) ? 1u : 0u;
                    cnsp = !spec;
                    mkray(ray, pos, eps, wn, 3.402823466e+38);
                    continue;
                }
                d3 fx, fy;
                frame(nrm, &fx, &fy);
                d3 lc = cos_hemi(u01(seed, vkey, 3), u01(seed, vkey, 4));
                if (!(lc.z > 0.0)) break;
                d3 wi = dnorm(dadd(dadd(dmul(fx, lc.x), dmul(fy, lc.y)), dmul(nrm, lc.z)));
                for (int c = 0; c < 3; c++) T[c] *= A[c];
                if (T[0] <= 0.0 && T[1] <= 0.0 && T[2] <= 0.0) break;
                if (i - 1 >= rr_start) {
                    double lum = 0.212671 * T[0] + 0.715160 * T[1] + 0.072169 * T[2];
                    double q = lum < rr_prob ? lum : rr_prob;
                    if (!(u01(seed, vkey, 5) < q)) break;
                    for (int c = 0; c < 3; c++) T[c] /= q;
                }
                cedges += cnsp ? 1u : 0u;
                cnsp = 1;
                mkray(ray, pos, eps, wi, 3.402823466e+38);
            }
            for (int c = 0; c < 3; c++) out_rgb[3 * ci + c] += L[c] / (double)n_iter;
        }
    }
    free(sparse);
    free(valid);
    free(dense);
    (void)nthreads;
}

/* ---- the reference's BDPT estimator (see rb2_oracle.h) ----------------------------- */
typedef struct { d3 pos, nrm, beta, wi, ng; uint32_t depth, mat; } ref_vertex;

/* One light subpath of the reference estimator; stores its vertices in
 * out[0 .. return value).  Keys: light salt, `key`. */
static uint32_t ref_light_path(const rb2o_bvh* b, const rb2o_scene* s, uint64_t ls, uint64_t key, uint32_t Dl,
                               ref_vertex* out)
{
    uint32_t j = (uint32_t)(u01(ls, key, 0) * s->n_lights);
    if (j >= s->n_lights) j = s->n_lights - 1;
    const uint32_t lt = s->lights[j];
    const uint32_t* lv = s->tris + 3 * (size_t)lt;
    d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
    double su = sqrt(u01(ls, key, 1)), u2 = u01(ls, key, 2);
    double b0 = 1.0 - su, b1 = u2 * su;
    d3 y0 = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
    d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
    /* DiffuseAreaLight::Le: uniform over the hemisphere about world +z, negated
     * when its dot product with the light normal is nonzero; Le / pdf with
     * pdf = (1 / area) (1 / 2 pi) / |cos|, Le only toward the front. */
    const double ln3[3] = {ln.x, ln.y, ln.z};
    double dir3[3], kk;
    /* compute_area (core/primitives.h:273-276) is 0.5 for every triangle. */
    rb2o_light_le_ref(ln3, 0.5, u01(ls, key, 3), u01(ls, key, 4), dir3, &kk);
    d3 dir = D3(dir3[0], dir3[1], dir3[2]);
    const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
    double beta[3] = {Le[0] * kk, Le[1] * kk, Le[2] * kk};
    float ray[8];
    mkray(ray, y0, 1.0e-4, dir, 3.402823466e+38);
    uint32_t nv = 0;
    for (uint32_t d = 1; d <= Dl; d++) {
        rb2o_hit h;
        trace_ct(b, ray, 0, &h, RB2O_RAY_LIGHT);
        if (h.prim < 0) break;
        const uint32_t* t = s->tris + 3 * (size_t)h.prim;
        const uint32_t m = s->tri_mat[h.prim];
        const float* E = s->emission + 3 * (size_t)m;
        const int emitter = E[0] > 0.0f || E[1] > 0.0f || E[2] > 0.0f;
        d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
        d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
        d3 dd = D3(ray[4], ray[5], ray[6]);
        d3 wo = dmul(dd, -1.0);
        d3 nrm = ddot(ng, wo) < 0.0 ? dmul(ng, -1.0) : ng;
        d3 pos = dadd(D3(ray[0], ray[1], ray[2]), dmul(dd, h.t));
        ref_vertex* V = &out[nv++];
        V->pos = pos; V->nrm = nrm; V->wi = wo; V->ng = ng; V->depth = d; V->mat = m;
        V->beta = emitter ? D3(0, 0, 0) : D3(beta[0], beta[1], beta[2]);
        if (emitter || d >= Dl) break;
        double fac[3];
        d3 wn;
        if (s->materials && !plain_lambertian(&s->materials[m])) {
            double pdf;
            int spec;
            d3 f = mat_sample(&s->materials[m], ng, wo, u01(ls, key, 8 + 8 * d), u01(ls, key, 9 + 8 * d),
                              u01(ls, key, 11 + 8 * d), &wn, &pdf, &spec, NULL);
            if (!(pdf > 0.0) || !(f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) break;
            double k = fabs(ddot(wn, ng)) / pdf;
            fac[0] = f.x * k; fac[1] = f.y * k; fac[2] = f.z * k;
        } else {
            d3 fx, fy;
            frame(nrm, &fx, &fy);
            d3 lc = cos_hemi(u01(ls, key, 8 + 8 * d), u01(ls, key, 9 + 8 * d));
            if (!(lc.z > 0.0)) break;
            wn = dnorm(dadd(dadd(dmul(fx, lc.x), dmul(fy, lc.y)), dmul(nrm, lc.z)));
            const float* A = s->albedo + 3 * (size_t)m;
            fac[0] = A[0]; fac[1] = A[1]; fac[2] = A[2];
        }
        double lum = 0.212671 * fac[0] + 0.715160 * fac[1] + 0.072169 * fac[2];
        double q = lum < 1.0 ? lum : 1.0;
        if (!(q > 0.0 && u01(ls, key, 10 + 8 * d) < q)) break;
        for (int cc = 0; cc < 3; cc++) beta[cc] *= fac[cc] / q;
        if (!(beta[0] > 0.0 || beta[1] > 0.0 || beta[2] > 0.0)) break;
        mkray(ray, pos, 1.0e-3 * (double)h.t, wn, 3.402823466e+38);
    }
    return nv;
}

void rb2o_bdpt_ref(const rb2o_bvh* b, const rb2o_scene* s, const float* cam_rays, uint32_t n_cam, uint32_t n_iter,
                   const rb2o_bdpt_ref_params* p, uint64_t seed, double* out_rgb, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    const uint32_t Dl = p->light_max_depth, NL = p->n_light_paths, C = p->connections;
    const uint32_t Kc = p->cam_max_depth + 1;
    const double inv_nl = s->n_lights ? 1.0 / (double)s->n_lights : 0.0;
    const uint64_t ls = seed ^ 0xA24BAED4963EE407ull;
    ref_vertex* sparse = (ref_vertex*)calloc((size_t)NL * Dl, sizeof(ref_vertex));
    uint32_t* nvert = (uint32_t*)calloc(NL, sizeof(uint32_t));
    ref_vertex* dense = (ref_vertex*)calloc((size_t)NL * Dl, sizeof(ref_vertex));
    for (size_t i = 0; i < (size_t)n_cam * 3; i++) out_rgb[i] = 0.0;
    /* Preparation pass: mean stored vertices per light subpath -> cache capacity. */
    uint64_t cap = (uint64_t)-1;
    if (p->n_prep > 0 && s->n_lights) {
        uint64_t total = 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
        {
            ref_vertex* tmp = (ref_vertex*)calloc(Dl, sizeof(ref_vertex));
            uint64_t part = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
            for (int64_t q = 0; q < (int64_t)p->n_prep; q++)
                part += ref_light_path(b, s, ls ^ 0x5EED5EED5EED5EEDull, (uint64_t)q, Dl, tmp);
#ifdef _OPENMP
#pragma omp atomic
#endif
            total += part;
            free(tmp);
        }
        float avg = (float)total / (float)p->n_prep;
        cap = (uint64_t)ceilf(1.1f * avg * (float)NL);
    }
    for (uint32_t it = 0; it < n_iter; it++) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
        for (int64_t q = 0; q < (int64_t)NL; q++)
            nvert[q] = s->n_lights ? ref_light_path(b, s, ls, (uint64_t)it * NL + (uint64_t)q, Dl, sparse + (size_t)q * Dl)
                                   : 0u;
        uint64_t M = 0;
        for (uint32_t q = 0; q < NL; q++)
            for (uint32_t k = 0; k < nvert[q]; k++)
                if (M < cap) dense[M++] = sparse[(size_t)q * Dl + k];
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
        for (int64_t ci = 0; ci < (int64_t)n_cam; ci++) {
            double L[3] = {0, 0, 0}, T[3] = {1, 1, 1};
            int prev_spec = 1; /* the camera counts as specular */
            float ray[8];
            for (int k = 0; k < 8; k++) ray[k] = cam_rays[8 * ((size_t)it * n_cam + ci) + k];
            const uint64_t key = (uint64_t)it * n_cam + (uint64_t)ci;
            for (uint32_t i = 1; i <= Kc; i++) {
                rb2o_hit h;
                trace_ct(b, ray, 0, &h, i == 1 ? RB2O_RAY_CAMERA : RB2O_RAY_EXTENSION);
                if (h.prim < 0) break;
                const uint32_t* t = s->tris + 3 * (size_t)h.prim;
                const uint32_t m = s->tri_mat[h.prim];
                d3 v0 = vtx(s, t[0]), v1 = vtx(s, t[1]), v2 = vtx(s, t[2]);
                d3 ng = dnorm(dcross(dsub(v1, v0), dsub(v2, v0)));
                d3 dd = D3(ray[4], ray[5], ray[6]);
                d3 wo = dmul(dd, -1.0);
                d3 pos = dadd(D3(ray[0], ray[1], ray[2]), dmul(dd, h.t));
                const double eps = 1.0e-3 * (double)h.t;
                const float* E = s->emission + 3 * (size_t)m;
                if (E[0] > 0.0f || E[1] > 0.0f || E[2] > 0.0f) {
                    if (prev_spec && ddot(ng, wo) > 0.0)
                        for (int c = 0; c < 3; c++) L[c] += T[c] * E[c];
                    break;
                }
                d3 nrm = ddot(ng, wo) < 0.0 ? dmul(ng, -1.0) : ng;
                const float* A = s->albedo + 3 * (size_t)m;
                const rb2o_material* mc = (s->materials && !plain_lambertian(&s->materials[m])) ? &s->materials[m] : NULL;
                frame3 frc = frame_z(ng);
                d3 wo_l = fr_local(&frc, wo);
                uint64_t vkey = key * 64 + i;
                uint64_t nkey = key * 64 + 1; /* NEE: the first vertex's draws at every vertex */
                if (s->n_lights) {
                    /* compute_direct_lighting (integrator_bdpt_lvc_sk.cu:233-327): a light
                     * sample and a BSDF sample toward one uniformly chosen emissive
                     * triangle j, balance-heuristic weights from the reference's pdfs
                     * (triangle area 0.5, no 1 / n_lights), the sum times n_lights. */
                    const double nl = (double)s->n_lights;
                    uint32_t j = (uint32_t)(u01(seed, nkey, 0) * s->n_lights);
                    if (j >= s->n_lights) j = s->n_lights - 1;
                    const uint32_t lt = s->lights[j];
                    const uint32_t* lv = s->tris + 3 * (size_t)lt;
                    d3 l0 = vtx(s, lv[0]), l1 = vtx(s, lv[1]), l2 = vtx(s, lv[2]);
                    d3 ln = dnorm(dcross(dsub(l1, l0), dsub(l2, l0)));
                    const float* Le = s->emission + 3 * (size_t)s->tri_mat[lt];
                    double su = sqrt(u01(seed, nkey, 1)), u2 = u01(seed, nkey, 2);
                    double b0 = 1.0 - su, b1 = u2 * su;
                    d3 lp = dadd(dadd(dmul(l0, b0), dmul(l1, b1)), dmul(l2, 1.0 - b0 - b1));
                    d3 dv = dsub(lp, pos);
                    double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                    d3 wi = dmul(dv, 1.0 / dist);
                    double cos_l = -ddot(ln, wi), cos_s = ddot(nrm, wi);
                    d3 f = D3(0, 0, 0);
                    double pdf_b = 0.0;
                    if (mc) {
                        d3 wi_l = fr_local(&frc, wi);
                        f = mat_f(mc, ng, wo, wi, wo_l, wi_l);
                        pdf_b = mat_pdf(mc, wo_l, wi_l);
                    } else if (cos_s > 0.0) {
                        f = dmul(D3(A[0], A[1], A[2]), 1.0 / RB2O_PI);
                        pdf_b = cos_s / RB2O_PI;
                    }
                    if (cos_l > 0.0 && dist > 0.0 && (f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) {
                        double pdf_l = dist2 / (0.5 * cos_l);
                        float sr[8];
                        mkray(sr, pos, eps, wi, dist * (1.0 - 1.0e-3));
                        if (!occluded(b, sr)) {
                            double k = fabs(cos_s) * (pdf_l / (pdf_l + pdf_b)) / pdf_l * nl;
                            L[0] += T[0] * f.x * Le[0] * k;
                            L[1] += T[1] * f.y * Le[1] * k;
                            L[2] += T[2] * f.z * Le[2] * k;
                        }
                    }
                    /* BSDF half: counts when the sampled ray's closest hit is triangle j. */
                    d3 wb = D3(0, 0, 0), fb = D3(0, 0, 0);
                    double pb = 0.0;
                    if (mc) {
                        int spec;
                        fb = mat_sample(mc, ng, wo, u01(seed, key, 8000), u01(seed, key, 8001), u01(seed, key, 8002),
                                        &wb, &pb, &spec, NULL);
                        if (spec) pb = 0.0;
                    } else {
                        d3 fx, fy;
                        frame(nrm, &fx, &fy);
                        d3 lc = cos_hemi(u01(seed, key, 8000), u01(seed, key, 8001));
                        if (lc.z > 0.0) {
                            wb = dnorm(dadd(dadd(dmul(fx, lc.x), dmul(fy, lc.y)), dmul(nrm, lc.z)));
                            fb = dmul(D3(A[0], A[1], A[2]), 1.0 / RB2O_PI);
                            pb = lc.z / RB2O_PI;
                        }
                    }
                    if (pb > 0.0 && (fb.x > 0.0 || fb.y > 0.0 || fb.z > 0.0)) {
                        /* sample_triangle_pdf: Moller-Trumbore of the ray against j. */
                        d3 e1 = dsub(l1, l0), e2 = dsub(l2, l0), pv = dcross(wb, e2);
                        double det = ddot(e1, pv);
                        if (!(det < 1.0e-6 && det > -1.0e-6)) {
                            d3 tv = dsub(pos, l0);
                            double uu = ddot(tv, pv) / det;
                            d3 qv = dcross(tv, e1);
                            double vv = ddot(wb, qv) / det, th = ddot(e2, qv) / det;
                            double cth = -ddot(ln, wb);
                            if (uu >= 0.0 && uu <= 1.0 && vv >= 0.0 && uu + vv <= 1.0 && th > eps && cth > 0.0) {
                                double pdf_l = th * th / (0.5 * cth);
                                float br[8];
                                mkray(br, pos, eps, wb, 3.402823466e+38);
                                rb2o_hit bh;
                                trace_ct(b, br, 0, &bh, RB2O_RAY_CONNECTION);
                                if (bh.prim == (int32_t)lt) {
                                    double k = fabs(ddot(wb, nrm)) * (pb / (pb + pdf_l)) / pb * nl;
                                    L[0] += T[0] * fb.x * Le[0] * k;
                                    L[1] += T[1] * fb.y * Le[1] * k;
                                    L[2] += T[2] * fb.z * Le[2] * k;
                                }
                            }
                        }
                    }
                }
                for (uint32_t cidx = 0; M > 0 && cidx < C; cidx++) {
                    uint64_t v = (uint64_t)(u01(seed, vkey, 16 + cidx) * (double)M);
                    if (v >= M) v = M - 1;
                    const ref_vertex* V = &dense[v];
                    d3 dv = dsub(V->pos, pos);
                    double dist2 = ddot(dv, dv), dist = sqrt(dist2);
                    if (!(dist > 0.0)) continue;
                    d3 dir = dmul(dv, 1.0 / dist);
                    double cos_c = ddot(nrm, dir), cos_v = -ddot(V->nrm, dir);
                    const rb2o_material* mv =
                        (s->materials && !plain_lambertian(&s->materials[V->mat])) ? &s->materials[V->mat] : NULL;
                    d3 fc = mc ? mat_f(mc, ng, wo, dir, wo_l, fr_local(&frc, dir))
                               : (cos_c > 0.0 ? dmul(D3(A[0], A[1], A[2]), 1.0 / RB2O_PI) : D3(0, 0, 0));
                    d3 fv;
                    if (mv) {
                        /* material_f(cached material, wo = toward the previous light
                         * vertex, wi = toward the camera vertex) */
                        frame3 frv = frame_z(V->ng);
                        d3 wiv = dmul(dir, -1.0);
                        fv = mat_f(mv, V->ng, V->wi, wiv, fr_local(&frv, V->wi), fr_local(&frv, wiv));
                    } else {
                        const float* Av = s->albedo + 3 * (size_t)V->mat;
                        fv = cos_v > 0.0 ? dmul(D3(Av[0], Av[1], Av[2]), 1.0 / RB2O_PI) : D3(0, 0, 0);
                    }
                    double g = fabs(cos_c) * fabs(cos_v) / dist2 / ((double)i + (double)V->depth);
                    double cv[3] = {T[0] * fc.x * fv.x * V->beta.x * g, T[1] * fc.y * fv.y * V->beta.y * g,
                                    T[2] * fc.z * fv.z * V->beta.z * g};
                    if (!(cv[0] > 0.0 || cv[1] > 0.0 || cv[2] > 0.0)) continue;
                    float cr[8];
                    mkray(cr, pos, eps, dir, dist * (1.0 - 1.0e-3));
                    if (occluded_t(b, cr, RB2O_RAY_CONNECTION)) continue;
                    for (int c = 0; c < 3; c++) L[c] += cv[c];
                }
                if (i >= Kc) break;
                d3 wn;
                int spec = 0;
                if (mc) {
                    double pdf;
                    d3 f = mat_sample(mc, ng, wo, u01(seed, vkey, 3), u01(seed, vkey, 4), u01(seed, vkey, 6), &wn, &pdf,
                                      &spec, NULL);
                    if (!(pdf > 0.0) || !(f.x > 0.0 || f.y > 0.0 || f.z > 0.0)) break;
                    double k = fabs(ddot(wn, ng)) / pdf;
                    T[0] *= f.x * k; T[1] *= f.y * k; T[2] *= f.z * k;
                } else {
                    d3 fx, fy;
                    frame(nrm, &fx, &fy);
                    d3 lc = cos_hemi(u01(seed, vkey, 3), u01(seed, vkey, 4));
                    if (!(lc.z > 0.0)) break;
                    wn = dnorm(dadd(dadd(dmul(fx, lc.x), dmul(fy, lc.y)), dmul(nrm, lc.z)));
                    for (int c = 0; c < 3; c++) T[c] *= A[c];
                }
                if (!(T[0] > 0.0 || T[1] > 0.0 || T[2] > 0.0)) break;
                if (!rr_step(T, i - 1, p->cam_rrstart, p->cam_rrprob, 2u, u01(seed, vkey, 5))) break;
                prev_spec = spec;
                mkray(ray, pos, eps, wn, 3.402823466e+38);
            }
            for (int c = 0; c < 3; c++) out_rgb[3 * ci + c] += L[c] / (double)n_iter;
        }
    }
    free(sparse);
    free(nvert);
    free(dense);
    (void)nthreads;
}
