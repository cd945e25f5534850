/*
 * TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's ray traversal,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The product library never includes, links or calls this.
 *
 * Parity pin: the traversal is restated from the reference's single-ray
 * trace_ray (accelerators/sbvh/cuda_tracer_functions.cu:42-279) and its span
 * helpers (accelerators/sbvh/cudatracerkernels.h:213-256).  The reference
 * ships no tests or golden vectors, so this restatement is pinned against the
 * reference's own host code compiled in place (oracle/_ref: SBVH builder,
 * Compact2 packer, camera, Moller-Trumbore) and against committed fixtures
 * generated from it (tests/golden/).
 */
#ifndef RB2_ORACLE_H
#define RB2_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int32_t prim; float t, u, v; } rb2o_hit;
typedef struct { uint32_t nodes, tris, leafterms, pad; } rb2o_counts;

/* Closest-hit / any-hit over Compact2 buffers (4 words per uint4).
 * rays: 8 floats per ray (ox, oy, oz, tmin, dx, dy, dz, tmax).
 * mask (nullable): rays with mask[i]==0 are skipped and report prim=-1.
 * counts (nullable): canonical single-lane visit counts per ray.
 * nthreads <= 0: use all OpenMP threads. */
void rb2o_trace(const uint32_t* nodes, const uint32_t* woop, const uint32_t* triidx,
                const float* rays, uint32_t n, int any_hit, const uint8_t* mask,
                rb2o_hit* out, rb2o_counts* counts, int nthreads);

/* Single Woop triangle test with the same arithmetic as the traversal.
 * Returns 1 and (t,u,v) when tmin < t < tmax and the barycentrics pass. */
int rb2o_woop_test(const uint32_t* woop12, const float* ray8, float tmax, float* tuv);

/* Brute force over every Woop triangle slot (closest accepted t; on equal t
 * the first slot wins).  Returns hit records with the original triangle id. */
void rb2o_bruteforce(const uint32_t* woop, const uint32_t* triidx, uint32_t n_woop_u4,
                     const float* rays, uint32_t n, rb2o_hit* out, int nthreads);

/* PCG32 (O'Neill 2014, pcg32_srandom_r / pcg32_random_r), the generator the
 * product uses for every seeded stream. */
typedef struct { uint64_t state, inc; } rb2o_pcg32;
void rb2o_pcg32_seed(rb2o_pcg32* r, uint64_t initstate, uint64_t initseq);
uint32_t rb2o_pcg32_next(rb2o_pcg32* r);

#ifdef __cplusplus
}
#endif
#endif
