/*
 * rb2.h -- C ABI of librb2, the B200 (sm_100a) ray-query engine that drops in
 * for renderbox2's acceleration-structure build, tracer and integrator path.
 *
 * Conventions
 *  - Every function returns an rb2_status (0 = RB2_OK); rb2_last_error() gives
 *    the thread-local text of the last failure.  Nothing asserts or aborts.
 *  - Pointers named d_* are device pointers on the tracer's device; h_* are
 *    host pointers.  Caller buffers are borrowed, never freed by the library.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Rays use the reference's Ray layout (core/primitives.h:145-208):
 *    two float4 per ray, (origin.xyz, tmin) then (direction.xyz, tmax).
 */
#ifndef RB2_H
#define RB2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RB2_OK = 0,
    RB2_EINVAL = 1,      /* bad argument */
    RB2_ENOMEM = 2,      /* host or device allocation failed */
    RB2_ECUDA = 3,       /* CUDA runtime error */
    RB2_EIO = 4,         /* file could not be read or written */
    RB2_EFORMAT = 5,     /* corrupt or unsupported BVH / cache contents */
    RB2_ETIMEOUT = 6,    /* a bounded wait ran out (device wait, or a served job's deadline) */
    RB2_EDEVICE = 7,     /* device-side check failed (status word set) */
    RB2_ENOTSUP = 8      /* feature not available on this device / build */
} rb2_status;

/* Node layouts (accelerators/sbvh/cudatracerkernels.h:85-90).  Only Compact2
 * (child index = float4 offset, the layout the reference's Kepler kernel
 * reads) is produced and traced. */
enum { RB2_LAYOUT_COMPACT = 0, RB2_LAYOUT_COMPACT2 = 1 };

const char* rb2_last_error(void);
const char* rb2_version(void);

/* ------------------------------------------------------------------ build --
 * Replaces BVH(Scene*, const Platform&, const BuildParams&)
 * (accelerators/sbvh/bvh.h:115) + CudaBvh(const BVH&, BVHLayout)
 * (accelerators/sbvh/cudabvh.h:80).  Defaults equal the reference's Platform
 * (accelerators/sbvh/platform.h:78-90) and BuildParams (bvh.h:104-112) and the
 * SplitBVHBuilder constants (splitbvhbuilder.h:135-140), except that the
 * number of spatial bins and the object-split binning threshold are tunable. */
typedef struct {
    float sah_node_cost;        /* 1.0 */
    float sah_triangle_cost;    /* 1.0 */
    uint32_t min_leaf_size;     /* 1 */
    uint32_t max_leaf_size;     /* 0x7FFFFFF */
    float split_alpha;          /* 1e-5: spatial split if child overlap >= alpha * root area */
    uint32_t max_depth;         /* 64 */
    uint32_t max_spatial_depth; /* 48 */
    uint32_t spatial_bins;      /* 64 (reference: 128) */
    uint32_t object_bins;       /* 64; nodes with <= exact_sweep_max refs use a full sorted sweep */
    uint32_t exact_sweep_max;   /* 512 */
    int32_t num_threads;        /* <= 0: all hardware threads */
    uint32_t layout;            /* RB2_LAYOUT_COMPACT2 */
} rb2_build_params;

typedef struct {
    uint64_t n_nodes_u4;        /* node buffer size in uint4 (4 per inner node) */
    uint64_t n_woop_u4;         /* Woop buffer size in uint4 (3 per tri ref + 1 per leaf) */
    uint64_t n_triidx;          /* == n_woop_u4 */
    uint32_t n_inner, n_leaves, n_tri_refs, n_tris;
    uint32_t max_depth;
    uint32_t layout;
    float sah;                  /* top-down SAH cost (bvnode.cpp:85-100 definition) */
    double build_ms;
} rb2_bvh_counts;

typedef struct rb2_host_bvh rb2_host_bvh;

int rb2_build_params_default(rb2_build_params* p);

/* v_xyz: nv vertices (float x,y,z); idx3: ntri triangles (3 vertex indices). */
int rb2_bvh_build(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri,
                  const rb2_build_params* params, rb2_host_bvh** out);

/* Wraps existing Compact2 buffers (e.g. from the reference's CudaBvh getters,
 * cudabvh.h:95-97).  The buffers are copied and validated. */
int rb2_bvh_from_buffers(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop,
                         uint64_t n_woop_u4, const uint32_t* triidx, uint64_t n_triidx,
                         rb2_host_bvh** out);

int rb2_bvh_counts_get(const rb2_host_bvh* b, rb2_bvh_counts* out);
/* Getters (cudabvh.h:95-97): pointers stay valid until rb2_host_bvh_free. */
const uint32_t* rb2_bvh_nodes(const rb2_host_bvh* b);
const uint32_t* rb2_bvh_woop(const rb2_host_bvh* b);
const uint32_t* rb2_bvh_triidx(const rb2_host_bvh* b);
void rb2_host_bvh_free(rb2_host_bvh* b);

/* BVH cache.  rb2_bvh_save writes the versioned binary format (magic "RB2BVH\0\1",
 * version, layout, counts, FNV-1a checksum).  rb2_bvh_load reads that format
 * or the reference's text cache (cudabvh.cpp:108-214, magic 0x76543210). */
int rb2_bvh_save(const rb2_host_bvh* b, const char* path);
int rb2_bvh_save_text(const rb2_host_bvh* b, const char* path);
int rb2_bvh_load(const char* path, rb2_host_bvh** out);

/* --------------------------------------------------------------- tracer --
 * Replaces CudaTracer(const CudaBvh&, MemoryAllocator&) (cudatracer.h:67) and
 * float trace(const RayBuffer&, IntersectionBuffer&, SceneBuffer&, uint8_t*
 * stencil, bool any_hit) (cudatracer.h:87). */
typedef struct rb2_tracer rb2_tracer;

typedef struct {
    int32_t prim;   /* original triangle index, -1 = miss */
    float t;        /* hit distance (tmax of the ray on a miss) */
    float u, v;     /* Woop barycentrics of the accepted triangle */
} rb2_hit;

/* Launch configuration of the persistent traversal kernel.  Zero fields mean
 * "use the tuned default". */
typedef struct {
    uint32_t block_threads;     /* threads per CTA: 64, 128 or 256 */
    uint32_t ctas_per_sm;       /* resident CTAs per SM (0 = occupancy maximum) */
    uint32_t fetch_threshold;   /* refill a warp when fewer lanes stay busy (reference: 20) */
    uint32_t regs;              /* register budget of the kernel variant: 64, 48 or 40 (0 = 64) */
    uint32_t node_threshold;    /* end a warp's node phase, and test the triangles its lanes hold,
                                   once fewer than this many lanes still traverse nodes (1..32;
                                   1 = only when none does, the reference's while-while; 0 = the
                                   layout's tuned default); results do not depend on it */
} rb2_launch_config;

/* Node layout of the bulk traversals: the reference's Compact2 buffer in its
 * DFS order (cudabvh.cpp:234-288), the same nodes breadth-first (top levels
 * contiguous), or a 4-wide layout collapsed from the binary tree (up to four
 * exact child boxes per 128-byte node; the same leaves and Woop triangles, so
 * hits are identical except which of two triangles at the same t is
 * reported), or a compressed 8-wide layout (RB2_NODE_ORDER_CW8: eight child
 * boxes quantized to 8 bits per plane in an 80-byte node, conservatively
 * enlarged, and the same Woop triangles stored per node; closest hits are
 * identical except for ties in t).  Integrators and rb2_trace_isect traverse
 * the compressed 8-wide layout when it is set and the binary Compact2 buffer
 * otherwise; rb2_tracer_dev_bvh (the header-only device traversal) always
 * uses the binary buffer. */
enum { RB2_NODE_ORDER_DFS = 0, RB2_NODE_ORDER_BFS = 1, RB2_NODE_ORDER_WIDE4 = 2, RB2_NODE_ORDER_CW8 = 3 };

/* Ray-query modes. */
enum { RB2_MODE_CLOSEST = 0, RB2_MODE_ANY = 1, RB2_MODE_OCCLUSION = 2 };

/* Uploads the BVH to the current CUDA device.  The tracer owns that memory. */
int rb2_tracer_create(const rb2_host_bvh* bvh, rb2_tracer** out);
int rb2_tracer_destroy(rb2_tracer* t);
int rb2_tracer_set_launch(rb2_tracer* t, const rb2_launch_config* cfg);
int rb2_tracer_device_bytes(const rb2_tracer* t, uint64_t* bytes);

/* Bulk trace of n rays (device buffers).  any_hit != 0 stops at the first
 * accepted triangle.  d_mask (nullable) is the reference's stencil: rays with
 * mask 0 are skipped and reported as misses.  Asynchronous on `stream`. */
int rb2_trace(rb2_tracer* t, const float* d_rays, uint32_t n, int any_hit, const uint8_t* d_mask,
              rb2_hit* d_hits, void* stream);

/* Device view of a tracer's BVH for kernels that call the header-only
 * rb2::trace_ray (rb2_device.cuh).  Replaces CudaTracer::get_bvh()
 * (cudatracer.h:89-101), which returned texture objects.  The pointers stay
 * valid until rb2_tracer_destroy. */
typedef struct {
    const void* nodes;        /* float4 Compact2 inner nodes, 16-byte aligned */
    const void* woop;         /* float4 Woop rows + terminators */
    const uint32_t* triidx;   /* original triangle id per Woop slot */
    uint64_t n_nodes_u4;
    uint64_t n_woop_u4;
} rb2_dev_bvh;
int rb2_tracer_dev_bvh(const rb2_tracer* t, rb2_dev_bvh* out);

/* Bulk trace with one thread per ray (no persistent queue) through the
 * header-only rb2::trace_ray: the pattern of kernels that trace inside their
 * own code, as the reference's integrator megakernels do
 * (integrators/integrator_path.cu:43-261 calls trace_ray).  Same outputs as
 * rb2_trace with single-lane traversal order. */
int rb2_trace_per_thread(rb2_tracer* t, const float* d_rays, uint32_t n, int any_hit, const uint8_t* d_mask,
                         rb2_hit* d_hits, void* stream);

/* Same from/to host memory: copies rays in, traces, copies hits out, and
 * synchronises `stream`.  Scratch device buffers are grown on demand and
 * reused across calls. */
int rb2_trace_host(rb2_tracer* t, const float* h_rays, uint32_t n, int any_hit, const uint8_t* h_mask,
                   rb2_hit* h_hits, void* stream);

/* Host-buffer traces of many jobs, pipelined: rays are cut into chunks that
 * cycle through `depth` streams, so the upload of one chunk, the traversal of
 * the previous one and the download of the one before overlap (copy engines
 * and SMs busy at once).  Host buffers should be pinned for the copies to be
 * asynchronous.  rb2_trace_host_jobs returns when every output is on the host;
 * its work starts after what is queued on `stream` and `stream` waits for all
 * of it (so CUDA events on `stream` bracket it).  The pipeline owns its
 * streams and device staging (depth x chunk x 49 B); one host thread at a time.
 * Extends the host-buffer path of rb2_trace_host (same outputs per job). */
typedef struct rb2_pipeline rb2_pipeline;
typedef struct {
    rb2_tracer* tracer;
    const float* h_rays;      /* 8 floats per ray */
    uint64_t n;
    uint32_t mode;            /* RB2_MODE_* (closest/any: rb2_hit out; occlusion: uint8 out) */
    uint32_t reserved;
    const uint8_t* h_mask;    /* nullable */
    void* h_out;
} rb2_host_job;
int rb2_pipeline_create(uint64_t chunk_rays, uint32_t depth, rb2_pipeline** out);
int rb2_pipeline_destroy(rb2_pipeline* p);
int rb2_trace_host_jobs(rb2_pipeline* p, const rb2_host_job* jobs, uint32_t n_jobs, void* stream);

/* Occlusion-only any-hit: writes 1 byte per ray (1 = occluded). */
int rb2_trace_occlusion(rb2_tracer* t, const float* d_rays, uint32_t n, const uint8_t* d_mask,
                        uint8_t* d_occluded, void* stream);

/* Device-side status word of the tracer (0 = clean).  Non-zero means a kernel
 * hit a guard (stack overflow on a corrupt tree, bad index) and skipped work. */
int rb2_tracer_status(rb2_tracer* t, uint32_t* status, void* stream);

/* Re-uploads the tracer's nodes in another order (RB2_NODE_ORDER_*); results
 * are unchanged, only memory locality differs.  Synchronises the device. */
int rb2_tracer_set_node_order(rb2_tracer* t, uint32_t order);
int rb2_tracer_get_node_order(const rb2_tracer* t, uint32_t* order);

/* The compressed 8-wide layout of a host BVH, as the tracer builds it for
 * RB2_NODE_ORDER_CW8, for tools and tests: call with NULL arrays for the
 * counts, then with arrays of n_nodes * 20, n_tris * 12 and n_tris words
 * (node words, Woop rows, original triangle ids). */
typedef struct {
    uint32_t n_nodes, n_tris, depth, reserved;
} rb2_cw8_counts;
int rb2_bvh_cw8_layout(const rb2_host_bvh* bvh, rb2_cw8_counts* counts, uint32_t* nodes, uint32_t* woop,
                       uint32_t* triidx);

/* -------------------------------------------------------------- batching --
 * Many scenes and ray batches of uneven size in ONE persistent launch: every
 * job's rays are served from a single global queue, so warps move between
 * scenes without a kernel boundary.  No reference counterpart (the reference
 * traces one RayBuffer per CudaTracer::trace call, cudatracer.cu:134-183). */
typedef struct {
    rb2_tracer* tracer;       /* scene (its device BVH) */
    const float* d_rays;      /* 2 float4 per ray, 16-byte aligned */
    uint64_t n;
    uint32_t mode;            /* RB2_MODE_* */
    uint32_t reserved;
    const uint8_t* d_mask;    /* nullable stencil */
    void* d_out;              /* rb2_hit[n] (closest/any) or uint8_t[n] (occlusion) */
} rb2_trace_job;

typedef struct {
    uint32_t block_threads;   /* 64, 128, 256 (0 = 128) */
    uint32_t ctas_per_sm;     /* 0 = occupancy maximum */
    uint32_t fetch_threshold; /* 0 = 20 */
    uint32_t chunk;           /* queue chunk: a warp reserves chunk*32 rays per atomic (0/1 = exact) */
    uint32_t node_order;      /* RB2_NODE_ORDER_*; applied to every tracer in the batch */
    uint32_t regs;            /* register budget of the kernel variant: 64, 48 or 40 (0 = 64);
                                 lower budgets keep more warps resident and spill a little to L1 */
    uint32_t reorder;         /* ray reordering before the traversal: 0 off, or k in 3..6: each job's
                                 rays are visited in the order of (direction octant, k-bit-per-axis
                                 Morton code of the origin within its scene's box), so a warp's rays
                                 start near each other and head the same way; records still go to
                                 each ray's own index, and every ray's result is unchanged */
    uint32_t node_threshold;  /* as rb2_launch_config.node_threshold (0 = the layout's default) */
} rb2_batch_config;

typedef struct rb2_batch rb2_batch;

/* Uploads the job table; buffers are borrowed and must outlive the batch. */
int rb2_batch_create(const rb2_trace_job* jobs, uint32_t n_jobs, rb2_batch** out);
int rb2_batch_destroy(rb2_batch* b);
int rb2_batch_set_config(rb2_batch* b, const rb2_batch_config* cfg);
int rb2_batch_get_config(const rb2_batch* b, rb2_batch_config* cfg);
/* Queue reset + one persistent kernel; replays the captured graph if any. */
int rb2_batch_launch(rb2_batch* b, void* stream);
/* Captures the launch (queue reset + kernel) into a CUDA graph on `stream`
 * (must be a non-default stream); later rb2_batch_launch calls replay it.
 * Changing the config drops the graph. */
int rb2_batch_capture(rb2_batch* b, void* stream);
int rb2_batch_status(rb2_batch* b, uint32_t* status, void* stream);
/* Times candidate configs (coordinate descent over node order, block shape x
 * register budget, node-phase threshold, CTAs per SM, fetch threshold and
 * queue chunk, without and with ray reordering; median of `reps` launches
 * each), applies and returns the fastest. */
int rb2_batch_autotune(rb2_batch* b, void* stream, uint32_t reps, rb2_batch_config* best, double* best_ms);

/* ------------------------------------------------------- fault injection --
 * Host-side hooks for tests of the error paths; no GPU fault is involved.
 * Every device allocation of the library goes through one wrapper.
 * rb2_debug_fail_alloc(k): the k-th device allocation from this call on
 * fails as cudaMalloc would when memory is exhausted (the entry point that
 * made it returns RB2_ENOMEM and frees what it had allocated); 0 disarms.
 * rb2_debug_alloc_count: successful allocations since load and allocations
 * not yet freed (for leak checks around create / destroy pairs). */
int rb2_debug_fail_alloc(uint64_t k);
int rb2_debug_alloc_count(uint64_t* total, int64_t* live);

/* --------------------------------------------------- allocation-free batch --
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory: hosts that own all device memory through their own
 * arena or admit work against a fixed memory budget, and loops in which
 * cudaMalloc/cudaFree, which can synchronise the device, must not appear.
 * The caller passes every input and output (BVH buffers, rays, results) in
 * memory it owns; the only scratch (job table, ray-count prefix, queue head,
 * status word) lives in a fixed file-scope device array of the library sized
 * for RB2_NOALLOC_MAX_JOBS jobs (about 18.5 KB, held on every GPU that loads
 * the library until the process exits).  This entry point calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *  - More than RB2_NOALLOC_MAX_JOBS jobs: returns RB2_EINVAL, nothing runs.
 *  - Every call reuses the same array (it keeps the last call's contents;
 *    the queue head and status are cleared at the start of each call), so
 *    calls whose work overlaps on the GPU race and corrupt each other:
 *    issue them one after another on one stream.
 *  - The first call on a device resolves the array's device address and the
 *    launch shape for that device (with that device current); make that first
 *    call before any stream capture on the device.
 *  - Buffers: d_nodes/d_woop/d_triidx are a Compact2 layout as produced by
 *    rb2_bvh_build or accepted by rb2_bvh_from_buffers, 16-byte aligned, and
 *    d_woop must stay readable for two uint4 past its last row. */
#define RB2_NOALLOC_MAX_JOBS 256

typedef struct {
    const float* d_nodes;     /* Compact2 nodes (uint4 words) */
    const float* d_woop;      /* Woop rows + 2 spare uint4 */
    const uint32_t* d_triidx; /* parallel to the Woop rows */
    const float* d_rays;      /* 2 float4 per ray */
    uint64_t n;
    uint32_t mode;            /* RB2_MODE_* */
    uint32_t reserved;
    const uint8_t* d_mask;    /* nullable stencil */
    void* d_out;              /* rb2_hit[n] (closest/any) or uint8_t[n] (occlusion) */
} rb2_noalloc_job;

int rb2_trace_batch_noalloc(const rb2_noalloc_job* jobs, uint32_t n_jobs, void* stream);
/* Guard bits of the last rb2_trace_batch_noalloc call that traced any ray on
 * the current device (0 = clean; bit 0 = a ray whose traversal stack would
 * have overflowed, as a corrupt or over-deep tree can cause, was reported as
 * a miss).  Copies the word from the shared array into *status on `stream`
 * and synchronises that stream; allocates nothing.  Issue it on the stream
 * of the trace call it checks, under the same one-stream rule. */
int rb2_trace_batch_noalloc_status(uint32_t* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RB2_H */
