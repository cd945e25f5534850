/*
 * rb2_serve.h -- continuous-batching serving runtime over resident BVHs.
 *
 * No reference counterpart: renderbox2 renders one configured scene per
 * process (core/application.cpp:100-239).  The server keeps a pool of BVHs,
 * device scenes and per-slot wavefront state resident on the device and
 * runs a real-time request loop: jobs (ray-query batches and path-traced
 * tiles) arrive at their timestamps, are admitted when an execution slot is
 * free and their device footprint fits the HBM budget, run concurrently on
 * the slots' streams (their kernels overlap on the GPU), and complete
 * asynchronously.  Latency = completion - arrival.  With fifo = 1 the same
 * loop runs one job at a time on one slot (the per-launch baseline).
 */
#ifndef RB2_SERVE_H
#define RB2_SERVE_H

#include "rb2.h"
#include "rb2_render.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { RB2_JOB_RAYS = 0, RB2_JOB_TILE = 1 };

typedef struct {
    uint32_t kind;          /* RB2_JOB_* */
    uint32_t bvh;           /* index into the server's resident pool */
    double arrival_s;       /* arrival time relative to the start of rb2_server_run */
    /* ray-query job */
    const float* h_rays;    /* host (pinned for speed): 8 floats per ray */
    uint64_t n_rays;
    uint32_t mode;          /* RB2_MODE_CLOSEST / RB2_MODE_ANY (rb2_hit out) or RB2_MODE_OCCLUSION (u8 out) */
    /* tile job: square path-traced image */
    uint32_t tile;          /* side in pixels */
    uint32_t spp, max_depth, rr_start;
    float rr_prob;
    uint64_t seed;
    float eye[3], lookat[3], up[3], fov_deg;
    void* h_out;            /* rays: rb2_hit[n] or uint8_t[n]; tile: float[tile*tile*3] mean radiance */
} rb2_job;

typedef struct {
    double admit_s, end_s, latency_s;
    uint64_t footprint_bytes;
    uint64_t rays;          /* rays traced for this job */
    uint32_t slot;
    int32_t status;         /* rb2_status of the job */
} rb2_job_result;

typedef struct {
    uint32_t slots;         /* concurrent execution slots (streams); 0 = 8, at most 256 (RB2_EINVAL above:
                               a tracer hands out 256 per-launch queue heads) */
    uint32_t fifo;          /* 1: one job at a time, arrival order, one slot */
    uint64_t hbm_budget;    /* bytes of job working set admitted at once; 0 = 8 GiB */
    uint32_t max_tile;      /* largest tile side (slot state is sized for it); 0 = 1024 */
    uint32_t job_timeout_ms;/* per-job deadline from admission; 0 = none.  A job still running at its
                               deadline gets status RB2_ETIMEOUT (latency = time to the deadline check)
                               and the loop goes on admitting and retiring other jobs; its slot and
                               budget share come back once its work has left the slot's stream, and
                               its output is unspecified.  rb2_server_run returns only after every
                               slot is idle, timed-out jobs included. */
    uint64_t max_rays;      /* largest ray job (slot staging); 0 = 4M */
} rb2_server_config;

typedef struct {
    double wall_s;
    uint64_t rays;
    double mrays_per_s;
    double p50_s, p99_s, mean_s, max_s;
    uint32_t max_concurrent;
    uint32_t jobs;
    uint64_t peak_admitted_bytes;
    uint64_t resident_bytes;  /* BVHs + scenes + slot state */
} rb2_server_stats;

typedef struct rb2_server rb2_server;

/* The pool arrays are borrowed and must outlive the server. */
int rb2_server_create(rb2_tracer* const* tracers, rb2_scene_dev* const* scenes, uint32_t n_bvh,
                      const rb2_server_config* cfg, rb2_server** out);
int rb2_server_destroy(rb2_server* s);
/* Runs the request loop until every job completed or timed out; results[i]
 * belongs to jobs[i].  Returns the first failing job's status (RB2_OK when
 * every job succeeded). */
int rb2_server_run(rb2_server* s, const rb2_job* jobs, uint32_t n_jobs, rb2_job_result* results,
                   rb2_server_stats* stats);
/* Device working set a job reserves against the HBM budget. */
uint64_t rb2_job_footprint(const rb2_job* job);

/* Fault injection on the host, for tests of the deadline: the next job the
 * loop enqueues waits behind a host function (cudaLaunchHostFunc) that
 * sleeps `ms` milliseconds on its slot's stream.  No GPU fault is involved. */
int rb2_debug_stall_next_job(uint32_t ms);

#ifdef __cplusplus
}
#endif
#endif
