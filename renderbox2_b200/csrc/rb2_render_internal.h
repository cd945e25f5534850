// Internal state of the device scene and the integrators, shared by the
// integrator kernels (rb2_render.cu) and the serving runtime (rb2_serve.cu).
#pragma once

#include "rb2.h"
#include "rb2_render.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace rb2dev {
struct MaterialDev;
}

struct rb2_scene_dev {
    float4* d_verts = nullptr;     // xyz, w unused
    uint4* d_tris = nullptr;       // vertex indices + material id
    float4* d_albedo = nullptr;    // per material
    float4* d_emission = nullptr;  // per material
    uint32_t* d_lights = nullptr;  // emissive triangle ids
    rb2dev::MaterialDev* d_mats = nullptr;  // layered materials (null: one Lambertian layer = albedo)
    bool layered = false;                   // some non-emitter material is not a single Lambertian layer
    uint32_t nv = 0, ntri = 0, n_mat = 0, n_lights = 0;
    uint64_t bytes = 0;
};

// Wavefront path state, one entry per path of the wave (SoA).
struct PathState {
    float4* T = nullptr;        // throughput rgb, w = solid-angle pdf of the last BSDF sample
    float4* L = nullptr;        // radiance gathered by the path
    float4* ray = nullptr;      // current extension ray (2 per path)
    int4* hit = nullptr;        // extension hit
    float4* sray = nullptr;     // pending shadow / connection ray (2 per path)
    float4* sc = nullptr;       // its contribution when unoccluded
    uint32_t* q[2] = {nullptr, nullptr};  // active-path queues (ping-pong)
    uint32_t* qs = nullptr;     // shadow queue
    uint64_t cap = 0;
};

// Device-side counters of one wave.
struct WaveCounters {
    uint32_t n_ext[2];
    uint32_t n_shadow;
    uint32_t n_conn;
    unsigned long long head_ext;     // traversal queue heads
    unsigned long long head_shadow;
    unsigned long long head_conn;
    unsigned long long stats[6];     // rb2_render_stats order
    uint32_t lvc_count;              // dense light-vertex-cache size of this iteration
    uint32_t pad;
};

// Light-vertex cache and light-path state of the BDPT integrator.
struct BdptState {
    // light subpaths
    float4* lray = nullptr;     // 2 per light path
    float4* lbeta = nullptr;    // throughput arriving at the next vertex
    int4* lhit = nullptr;
    uint32_t* lq[2] = {nullptr, nullptr};
    uint64_t cap_paths = 0;
    // cache: sparse (path, depth) slots and the dense list of valid slot indices
    float4* s_pos = nullptr;    // xyz, w = light-subpath vertex count s (as float)
    float4* s_nrm = nullptr;    // normal facing the arriving light, w = material id bits
    float4* s_beta = nullptr;
    float4* s_wi = nullptr;     // toward the previous light vertex, w = sign of ng . nrm
    uint8_t* s_valid = nullptr;
    uint32_t* d_slot = nullptr;    // valid slots in slot order (the compacted cache)
    uint32_t* block_sums = nullptr;
    uint64_t cap_slots = 0;
    uint32_t* lvc_off = nullptr;   // dense-cache offset of each iteration of a wave (kMaxBdptWave + 1)
    // connection rays of camera vertices (connections per path)
    float4* cray = nullptr;
    float4* cc = nullptr;
    uint32_t* cq = nullptr;
    uint64_t cap_conn = 0;
};

struct rb2_integrator {
    rb2_tracer* tracer = nullptr;
    const rb2_scene_dev* scene = nullptr;
    int sms = 0;
    // launch shape of the integrator's traversal kernels (rb2_integrator_set_launch)
    uint32_t tr_block = 128, tr_regs = 0, tr_threshold = 24;   // tr_regs 0: 48 binary, 64 compressed 8-wide
    uint32_t tr_node_threshold = 0;                             // 0: the layout's default
    // paths in flight per wave (rb2_integrator_set_wave; 0: the defaults below)
    uint64_t wave_paths = 0;
    // traversal timing (rb2_integrator_set_timing): an event pair per launch
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    uint32_t ev_used = 0;
    // generic scratch
    float4* d_rays = nullptr; uint64_t cap_rays = 0;        // 2 per ray
    int4* d_hits = nullptr; uint64_t cap_hits = 0;
    uint32_t* d_count = nullptr; uint64_t cap_count = 0;
    unsigned long long* d_counters = nullptr;                // queue heads (16)
    float4* d_accum = nullptr; uint64_t cap_accum = 0;
    float2* d_film_xy = nullptr; uint64_t cap_film_xy = 0;  // sample raster positions (filtered film)
    rb2_filter filter{RB2_FILTER_NONE, 0.5f, 0.5f, 0.0f};
    PathState ps;
    BdptState bd;
    WaveCounters* d_wave = nullptr;
    uint64_t bytes() const
    {
        return cap_rays * 32 + cap_hits * 16 + cap_count * 4 + 16 * 8 + cap_accum * 16 + cap_film_xy * 8 +
               ps.cap * (16 * 8 + 12) +
               sizeof(WaveCounters) + bd.cap_paths * (32 + 16 + 16 + 8) + bd.cap_slots * (4 * 16 + 1 + 4) +
               bd.cap_conn * (32 + 16 + 4);
    }
};

namespace rb2dev {
struct FilmArgs;
}

namespace rb2 {
// Kernel arguments of the film gather for a validated filter (rb2_film.cu).
int film_args(const rb2_filter& f, uint32_t width, uint32_t height, rb2dev::FilmArgs& out);

// Allocates (or grows) the wavefront path state / cache / connection buffers.
int ensure_path_state(PathState& ps, uint64_t P);
int ensure_bdpt_state(BdptState& bd, uint64_t n_paths, uint64_t n_slots, uint64_t n_conn);
// Grows an integrator's path-tracing scratch so renders of up to `paths`
// paths in flight and `npix` pixels run without further device allocation.
int integrator_reserve_pt(rb2_integrator* it, uint64_t paths, uint64_t npix);
// Paths in flight that rb2_render_pt uses for an image of npix pixels at spp.
// Paths in flight of a path-traced render: npix x spp_per_wave, or (0) as
// many samples per pixel as fit `auto_paths` (at least one, at most spp).
// Renders default to 32M paths (about 4.4 GB of path state): on config 2,
// 8M paths per wave measured 469 ms a frame, 16M 452 ms, 32M 445 ms (fewer
// launch tails).  Serving slots size for 8M so a slot stays about 1.1 GB.
constexpr uint64_t kRenderWavePaths = 32ull << 20;
constexpr uint64_t kServeWavePaths = 8ull << 20;
// BDPT runs several iterations (one camera sample per pixel each) per wave:
// as many as fit 8M camera paths, at most kMaxBdptWave.  Config 3 (921,600
// pixels, 16 iterations) measured 163 ms a frame one iteration at a time and
// about 125-130 ms with 4-16 in flight: the traversal launches grow from
// 0.9M to several million rays and their tails shrink in proportion.
constexpr uint64_t kBdptWavePaths = 8ull << 20;
constexpr uint32_t kMaxBdptWave = 64;
uint64_t pt_paths_in_flight(uint64_t npix, uint32_t spp, uint32_t spp_per_wave, uint64_t auto_paths = kRenderWavePaths);
}  // namespace rb2
