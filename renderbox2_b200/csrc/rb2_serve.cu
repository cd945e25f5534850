// Continuous-batching serving runtime (see include/rb2_serve.h).
//
// Slots are CUDA streams, each with resident state sized for the largest job
// it may run: ray staging buffers and an integrator whose path-tracing scratch
// is reserved up front, so the request loop never allocates device memory.
// The loop admits arriving jobs in arrival order while a slot is free and the
// admitted working sets fit the HBM budget, enqueues each job's copies and
// kernels on its slot's stream, and retires jobs by polling their completion
// events; kernels of different slots run concurrently on the GPU.
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_internal.h"
#include "rb2_render.h"
#include "rb2_render_internal.h"
#include "rb2_serve.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <numeric>
#include <thread>
#include <vector>

using namespace rb2;

namespace {

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    rb2_integrator* it = nullptr;
    float4* d_rays = nullptr;
    int4* d_out = nullptr;   // rb2_hit or uint8 occlusion
    float* d_img = nullptr;
    int job = -1;           // job running on the slot, -1 = none
    bool draining = false;  // a timed-out job's work is still on the stream
    double deadline = 0.0;  // loop time after which the running job times out
    uint64_t footprint = 0; // bytes the slot holds against the HBM budget
};

uint64_t out_bytes_per_ray(uint32_t mode) { return mode == RB2_MODE_OCCLUSION ? 1 : 16; }

// Host-side fault injection (rb2_debug_stall_next_job): the next enqueued job
// waits behind a host function that sleeps this many milliseconds.
std::atomic<uint32_t> g_stall_next_ms{0};

void CUDART_CB sleep_host_fn(void* ms)
{
    std::this_thread::sleep_for(std::chrono::milliseconds((uintptr_t)ms));
}

}  // namespace

struct rb2_server {
    std::vector<rb2_tracer*> tracers;
    std::vector<rb2_scene_dev*> scenes;
    rb2_server_config cfg{};
    std::vector<Slot> slots;
    uint64_t resident = 0;
};

extern "C" uint64_t rb2_job_footprint(const rb2_job* j)
{
    if (!j) return 0;
    if (j->kind == RB2_JOB_RAYS) return j->n_rays * (32 + out_bytes_per_ray(j->mode));
    const uint64_t npix = (uint64_t)j->tile * j->tile;
    const uint64_t P = pt_paths_in_flight(npix, j->spp, 0, kServeWavePaths);
    // path state (T, L, ray, hit, shadow ray, contribution, three queues) + accumulator + image
    return P * (16 + 16 + 32 + 16 + 32 + 16 + 12) + npix * (16 + 12) + sizeof(WaveCounters);
}

extern "C" int rb2_server_destroy(rb2_server* s)
{
    if (!s) return RB2_OK;
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        rb2_integrator_destroy(sl.it);
        rb2::dev_free(sl.d_rays);
        rb2::dev_free(sl.d_out);
        rb2::dev_free(sl.d_img);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    delete s;
    return RB2_OK;
}

extern "C" int rb2_server_create(rb2_tracer* const* tracers, rb2_scene_dev* const* scenes, uint32_t n_bvh,
                                 const rb2_server_config* cfg, rb2_server** out)
{
    if (!tracers || !scenes || !out || n_bvh == 0) return fail(RB2_EINVAL, "server needs a non-empty BVH pool");
    *out = nullptr;
    for (uint32_t i = 0; i < n_bvh; i++)
        if (!tracers[i] || !scenes[i]) return fail(RB2_EINVAL, "null tracer or scene in the pool");
    std::unique_ptr<rb2_server> s(new rb2_server());
    s->tracers.assign(tracers, tracers + n_bvh);
    s->scenes.assign(scenes, scenes + n_bvh);
    if (cfg) s->cfg = *cfg;
    rb2_server_config& c = s->cfg;
    if (!c.slots) c.slots = 8;
    if (c.fifo) c.slots = 1;
    if (!c.hbm_budget) c.hbm_budget = 8ull << 30;
    if (!c.max_tile) c.max_tile = 1024;
    if (!c.max_rays) c.max_rays = 4ull << 20;
    // Ray jobs take their queue head from the tracer's ring of per-launch
    // counters; more slots than ring entries could hand two concurrent
    // launches the same head.
    if (c.slots > kTracerQueueSlots)
        return fail(RB2_EINVAL, "at most " + std::to_string(kTracerQueueSlots) + " server slots");
    if (c.max_rays > 0xFFFFFFFFull) return fail(RB2_EINVAL, "max_rays must fit 32 bits");
    const uint64_t max_npix = (uint64_t)c.max_tile * c.max_tile;
    // Path state for the largest tile at up to 64 spp in flight (larger spp
    // counts stream through the same state in waves).
    const uint64_t max_paths = pt_paths_in_flight(max_npix, 64, 0, kServeWavePaths);
    for (uint64_t i = 0; i < n_bvh; i++) {
        uint64_t b = 0;
        rb2_tracer_device_bytes(tracers[i], &b);
        s->resident += b;
        rb2_scene_device_bytes(scenes[i], &b);
        s->resident += b;
    }
    s->slots.resize(c.slots);
    for (Slot& sl : s->slots) {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = rb2::dev_malloc(&sl.d_rays, c.max_rays * 32)) != cudaSuccess ||
            (e = rb2::dev_malloc(&sl.d_out, c.max_rays * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&sl.d_img, max_npix * 12)) != cudaSuccess) {
            rb2_server_destroy(s.release());
            return fail(RB2_ENOMEM, std::string("server slot: ") + cudaGetErrorString(e));
        }
        int rc = rb2_integrator_create(tracers[0], scenes[0], &sl.it);
        if (!rc) rc = integrator_reserve_pt(sl.it, max_paths, max_npix);
        if (rc) {
            rb2_server_destroy(s.release());
            return rc;
        }
        uint64_t b = 0;
        rb2_integrator_device_bytes(sl.it, &b);
        s->resident += b + c.max_rays * 48 + max_npix * 12;
    }
    *out = s.release();
    return RB2_OK;
}

namespace {

int enqueue(rb2_server* s, Slot& sl, const rb2_job& j)
{
    cudaStream_t st = sl.stream;
    if (j.bvh >= s->tracers.size()) return fail(RB2_EINVAL, "job names a BVH outside the pool");
    if (const uint32_t ms = g_stall_next_ms.exchange(0)) {
        cudaError_t e = cudaLaunchHostFunc(st, sleep_host_fn, (void*)(uintptr_t)ms);
        if (e != cudaSuccess) return fail(RB2_ECUDA, std::string("stall injection: ") + cudaGetErrorString(e));
    }
    if (j.kind == RB2_JOB_RAYS) {
        if (j.n_rays > s->cfg.max_rays || (j.n_rays && (!j.h_rays || !j.h_out)) || j.mode > RB2_MODE_OCCLUSION)
            return fail(RB2_EINVAL, "bad ray job");
        if (j.n_rays == 0) return RB2_OK;
        cudaError_t e = cudaMemcpyAsync(sl.d_rays, j.h_rays, j.n_rays * 32, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(RB2_ECUDA, std::string("job upload: ") + cudaGetErrorString(e));
        int rc = j.mode == RB2_MODE_OCCLUSION
                     ? rb2_trace_occlusion(s->tracers[j.bvh], reinterpret_cast<const float*>(sl.d_rays),
                                           (uint32_t)j.n_rays, nullptr, reinterpret_cast<uint8_t*>(sl.d_out), st)
                     : rb2_trace(s->tracers[j.bvh], reinterpret_cast<const float*>(sl.d_rays), (uint32_t)j.n_rays,
                                 j.mode == RB2_MODE_ANY, nullptr, reinterpret_cast<rb2_hit*>(sl.d_out), st);
        if (rc) return rc;
        e = cudaMemcpyAsync(j.h_out, sl.d_out, j.n_rays * out_bytes_per_ray(j.mode), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return fail(RB2_ECUDA, std::string("job download: ") + cudaGetErrorString(e));
        return RB2_OK;
    }
    if (j.kind != RB2_JOB_TILE) return fail(RB2_EINVAL, "unknown job kind");
    if (j.tile == 0 || j.tile > s->cfg.max_tile || !j.h_out || j.spp == 0) return fail(RB2_EINVAL, "bad tile job");
    sl.it->tracer = s->tracers[j.bvh];
    sl.it->scene = s->scenes[j.bvh];
    rb2_camera cam;
    int rc = rb2_camera_init(&cam, j.eye, j.lookat, j.up, j.tile, j.tile, j.fov_deg);
    if (rc) return rc;
    // The slot's path state was reserved for the serving wave size.
    const uint64_t npix = (uint64_t)j.tile * j.tile;
    const uint32_t spw = (uint32_t)(pt_paths_in_flight(npix, j.spp, 0, kServeWavePaths) / npix);
    rb2_pt_params p{j.spp, j.max_depth, j.rr_start, j.rr_prob, j.seed, spw, 0};
    if ((rc = rb2_render_pt(sl.it, &cam, &p, sl.d_img, st))) return rc;
    cudaError_t e = cudaMemcpyAsync(j.h_out, sl.d_img, (size_t)j.tile * j.tile * 12, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return fail(RB2_ECUDA, std::string("tile download: ") + cudaGetErrorString(e));
    return RB2_OK;
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" int rb2_server_run(rb2_server* s, const rb2_job* jobs, uint32_t n_jobs, rb2_job_result* results,
                              rb2_server_stats* stats)
{
    rb2::Range nvtx_range("rb2_server_run");
    if (!s || (n_jobs && (!jobs || !results))) return fail(RB2_EINVAL, "null argument");
    for (Slot& sl : s->slots) {
        sl.job = -1;
        sl.draining = false;
        sl.footprint = 0;
    }
    const double timeout_s = s->cfg.job_timeout_ms ? s->cfg.job_timeout_ms * 1e-3 : 0.0;
    std::vector<uint32_t> order(n_jobs);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
    for (uint32_t i = 0; i < n_jobs; i++) results[i] = rb2_job_result{};
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    uint32_t next = 0, done = 0, active = 0, max_active = 0;
    uint64_t admitted = 0, peak = 0;
    int first_error = RB2_OK;
    while (done < n_jobs) {
        bool progress = false;
        // Retire finished jobs; time out jobs past their deadline.
        for (uint32_t k = 0; k < s->slots.size(); k++) {
            Slot& sl = s->slots[k];
            if (sl.draining) {
                // The timed-out job's work has left the stream: the slot and
                // its share of the budget are free again.
                if (cudaEventQuery(sl.done) == cudaErrorNotReady) continue;
                sl.draining = false;
                admitted -= sl.footprint;
                sl.footprint = 0;
                progress = true;
                continue;
            }
            if (sl.job < 0) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) {
                if (timeout_s > 0.0 && now() > sl.deadline) {
                    rb2_job_result& r = results[sl.job];
                    r.end_s = now();
                    r.latency_s = r.end_s - jobs[sl.job].arrival_s;
                    r.status = fail(RB2_ETIMEOUT, "job " + std::to_string(sl.job) + " passed its " +
                                                      std::to_string(s->cfg.job_timeout_ms) + " ms deadline");
                    if (!first_error) first_error = r.status;
                    sl.job = -1;
                    sl.draining = true;
                    active--;
                    done++;
                    progress = true;
                }
                continue;
            }
            rb2_job_result& r = results[sl.job];
            const rb2_job& j = jobs[sl.job];
            r.end_s = now();
            r.latency_s = r.end_s - j.arrival_s;
            if (q != cudaSuccess) {
                r.status = fail(RB2_ECUDA, std::string("job failed: ") + cudaGetErrorString(q));
                if (!first_error) first_error = r.status;
            }
            if (j.kind == RB2_JOB_RAYS) {
                r.rays = j.n_rays;
            } else {
                rb2_render_stats rs;
                if (rb2_integrator_stats(sl.it, &rs, sl.stream) == RB2_OK)
                    r.rays = rs.primary_rays + rs.extension_rays + rs.shadow_rays;
            }
            admitted -= sl.footprint;
            sl.footprint = 0;
            sl.job = -1;
            active--;
            done++;
            progress = true;
        }
        // Admit arrived jobs in arrival order.
        const double t = now();
        while (next < n_jobs && jobs[order[next]].arrival_s <= t) {
            const uint32_t ji = order[next];
            const uint64_t fp = rb2_job_footprint(&jobs[ji]);
            if (active > 0 && admitted + fp > s->cfg.hbm_budget) break;  // wait for memory
            Slot* free_slot = nullptr;
            uint32_t slot_idx = 0;
            for (uint32_t k = 0; k < s->slots.size(); k++)
                if (s->slots[k].job < 0 && !s->slots[k].draining) { free_slot = &s->slots[k]; slot_idx = k; break; }
            if (!free_slot) break;  // wait for a slot
            rb2_job_result& r = results[ji];
            r.admit_s = t;
            r.footprint_bytes = fp;
            r.slot = slot_idx;
            const int rc = enqueue(s, *free_slot, jobs[ji]);
            next++;
            progress = true;
            if (rc) {
                r.status = rc;
                r.end_s = now();
                r.latency_s = r.end_s - jobs[ji].arrival_s;
                if (!first_error) first_error = rc;
                done++;
                continue;
            }
            cudaEventRecord(free_slot->done, free_slot->stream);
            free_slot->job = (int)ji;
            free_slot->deadline = t + timeout_s;
            free_slot->footprint = fp;
            admitted += fp;
            peak = std::max(peak, admitted);
            active++;
            max_active = std::max(max_active, active);
        }
        if (!progress) {
            // Nothing to retire or admit: wait briefly for the next arrival or completion.
            const double wait = next < n_jobs ? jobs[order[next]].arrival_s - now() : 0.0;
            if (active == 0 && wait > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(wait - 1e-4));
            else std::this_thread::yield();
        }
    }
    // Timed-out jobs may still be writing their outputs: return only once
    // every slot's stream is idle.
    for (Slot& sl : s->slots) {
        if (sl.draining) cudaEventSynchronize(sl.done);
        sl.draining = false;
        sl.footprint = 0;
    }
    const double wall = now();
    if (stats) {
        std::vector<double> lat(n_jobs);
        uint64_t rays = 0;
        double sum = 0.0, mx = 0.0;
        for (uint32_t i = 0; i < n_jobs; i++) {
            lat[i] = results[i].latency_s;
            rays += results[i].rays;
            sum += lat[i];
            mx = std::max(mx, lat[i]);
        }
        stats->wall_s = wall;
        stats->rays = rays;
        stats->mrays_per_s = wall > 0 ? (double)rays / wall / 1e6 : 0.0;
        stats->p50_s = percentile(lat, 0.50);
        stats->p99_s = percentile(lat, 0.99);
        stats->mean_s = n_jobs ? sum / n_jobs : 0.0;
        stats->max_s = mx;
        stats->max_concurrent = max_active;
        stats->jobs = n_jobs;
        stats->peak_admitted_bytes = peak;
        stats->resident_bytes = s->resident;
    }
    return first_error;
}

extern "C" int rb2_debug_stall_next_job(uint32_t ms)
{
    g_stall_next_ms.store(ms);
    return RB2_OK;
}
