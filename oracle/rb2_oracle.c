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

#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RB2O_SENTINEL 0x76543210
#define RB2O_STACK 64

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
