// Tracer (device BVH) and the bulk / batched traversal entry points, plus
// camera-ray generation.
//
// Every traversal launch runs k_trace_jobs<BLOCK> (rb2_sources.cuh), the
// persistent while-while kernel of rb2_traverse.cuh: a single-scene trace is a
// one-entry job table passed inline; a batch serves many (scene, ray batch,
// mode) jobs from one queue in one launch, optionally replayed from a CUDA
// graph.  B200 specifics: LDG.128 non-coherent loads instead of texture
// objects, full-warp *_sync votes, a queue counter per launch slot (so traces
// on different streams never share a counter; the reference's global
// g_warpCounter made trace() non-reentrant, kepler_dynamic_fetch.h:65), and a
// stack guard that records a status bit instead of writing out of bounds.
#include "rb2.h"
#include "rb2_devmem.h"
#include "rb2_internal.h"
#include "rb2_render.h"
#include "rb2_sources.cuh"
#include "rb2_camera.cuh"
#include "rb2_reorder.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <mutex>

namespace rb2 {
const HostBvh& host_of(const rb2_host_bvh* b);
}

namespace rb2dev {

__global__ void k_camera_rays(CamArgs c, float4* rays)
{
    const uint64_t total = (uint64_t)c.width * c.height * c.spp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pix = i / c.spp;
        const uint32_t px = (uint32_t)(pix % c.width), py = (uint32_t)(pix / c.width);
        float jx = 0.5f, jy = 0.5f;
        if (c.jitter) {
            uint64_t key = (c.seed * 0x9E3779B97F4A7C15ULL) ^ (i * 2ULL);
            jx = (float)(pcg_hash(key) >> 8) * (1.0f / 16777216.0f);
            jy = (float)(pcg_hash(key + 1) >> 8) * (1.0f / 16777216.0f);
        }
        float4 o, d;
        camera_ray(c.r2c, c.c2w, (float)px + jx, (float)py + jy, o, d);
        rays[2 * i + 0] = o;
        rays[2 * i + 1] = d;
    }
}

__global__ void k_camera_rays_at(CamArgs c, const float2* xy, uint32_t n, float4* rays)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 o, d;
        const float2 p = xy[i];
        camera_ray(c.r2c, c.c2w, p.x, p.y, o, d);
        rays[2 * (size_t)i + 0] = o;
        rays[2 * (size_t)i + 1] = d;
    }
}

}  // namespace rb2dev

// ======================================================================= host side
using namespace rb2;

namespace {

constexpr uint32_t kSlots = kTracerQueueSlots;
constexpr uint32_t kDefaultBlock = 128;

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(rb2::cuda_status(e), std::string(what) + ": " + cudaGetErrorString(e));
}

#define RB2_CUDA(call, what)                                \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);  \
    } while (0)

// Kernel variants: block shape {64, 128, 256} x register budget {64, 48, 40}
// x node layout {binary, 4-wide, compressed 8-wide}.
struct Occupancy {
    int sms = 0;
    int per_sm[3][3][3] = {};  // [block index][register-budget index][rb2dev::Layout]
};

// Kernel layout of a node order.
int layout_of(uint32_t node_order)
{
    return node_order == RB2_NODE_ORDER_WIDE4 ? rb2dev::kLayoutWide4
                                              : (node_order == RB2_NODE_ORDER_CW8 ? rb2dev::kLayoutCw8 : rb2dev::kLayoutBinary);
}

int block_index(uint32_t block) { return block == 64 ? 0 : (block == 256 ? 2 : 1); }
int regs_index(uint32_t regs) { return regs == 48 ? 1 : (regs == 40 ? 2 : 0); }

template <int B, int R>
int occ_of(int* out, size_t smem)
{
    RB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&out[0], rb2dev::k_trace_jobs<B, R, rb2dev::kLayoutBinary>, B, smem),
             "occupancy");
    RB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&out[1], rb2dev::k_trace_jobs<B, R, rb2dev::kLayoutWide4>, B, smem),
             "occupancy");
    RB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&out[2], rb2dev::k_trace_jobs<B, R, rb2dev::kLayoutCw8>, B, smem),
             "occupancy");
    return RB2_OK;
}

int occupancy(Occupancy& o)
{
    int dev = 0;
    RB2_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    RB2_CUDA(cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    const size_t smem = rb2dev::job_smem_bytes(rb2dev::kMaxSmemJobs, false);
    int rc = 0;
    rc |= occ_of<64, 64>(o.per_sm[0][0], smem) | occ_of<64, 48>(o.per_sm[0][1], smem) | occ_of<64, 40>(o.per_sm[0][2], smem);
    rc |= occ_of<128, 64>(o.per_sm[1][0], smem) | occ_of<128, 48>(o.per_sm[1][1], smem) | occ_of<128, 40>(o.per_sm[1][2], smem);
    rc |= occ_of<256, 64>(o.per_sm[2][0], smem) | occ_of<256, 48>(o.per_sm[2][1], smem) | occ_of<256, 40>(o.per_sm[2][2], smem);
    return rc ? RB2_ECUDA : RB2_OK;
}

template <int B, int R, int W>
void launch_variant(const rb2dev::KernelArgs& a, unsigned blocks, size_t smem, cudaStream_t s)
{
    rb2dev::k_trace_jobs<B, R, W><<<blocks, B, smem, s>>>(a);
}

template <int W>
void launch_shape(int variant, const rb2dev::KernelArgs& a, unsigned g, size_t smem, cudaStream_t s)
{
    switch (variant) {
    case 0: launch_variant<64, 64, W>(a, g, smem, s); break;
    case 1: launch_variant<64, 48, W>(a, g, smem, s); break;
    case 2: launch_variant<64, 40, W>(a, g, smem, s); break;
    case 4: launch_variant<128, 48, W>(a, g, smem, s); break;
    case 5: launch_variant<128, 40, W>(a, g, smem, s); break;
    case 6: launch_variant<256, 64, W>(a, g, smem, s); break;
    case 7: launch_variant<256, 48, W>(a, g, smem, s); break;
    case 8: launch_variant<256, 40, W>(a, g, smem, s); break;
    default: launch_variant<128, 64, W>(a, g, smem, s); break;
    }
}

// Launches the persistent kernel: grid = SMs x resident CTAs per SM, capped
// by the work available.
int launch_jobs(const rb2dev::KernelArgs& a, uint64_t total_rays, uint32_t block, uint32_t ctas_per_sm, uint32_t regs,
                int layout, const Occupancy& occ, cudaStream_t s)
{
    const int bi = block_index(block), ri = regs_index(regs);
    const int max_per_sm = std::max(1, occ.per_sm[bi][ri][layout]);
    const uint32_t per_sm = ctas_per_sm ? std::min<uint32_t>(ctas_per_sm, (uint32_t)max_per_sm) : (uint32_t)max_per_sm;
    uint64_t blocks = (uint64_t)occ.sms * per_sm;
    const uint64_t warps_needed = (total_rays + 31) / 32;
    const uint32_t bthreads = bi == 0 ? 64 : (bi == 2 ? 256 : 128);
    blocks = std::min<uint64_t>(blocks, (warps_needed + bthreads / 32 - 1) / (bthreads / 32));
    blocks = std::max<uint64_t>(blocks, 1);
    const size_t smem = rb2dev::job_smem_bytes(a.n_jobs, a.jobs == nullptr);
    if (layout == rb2dev::kLayoutWide4) launch_shape<rb2dev::kLayoutWide4>(bi * 3 + ri, a, (unsigned)blocks, smem, s);
    else if (layout == rb2dev::kLayoutCw8) launch_shape<rb2dev::kLayoutCw8>(bi * 3 + ri, a, (unsigned)blocks, smem, s);
    else launch_shape<rb2dev::kLayoutBinary>(bi * 3 + ri, a, (unsigned)blocks, smem, s);
    RB2_CUDA(cudaGetLastError(), "trace launch");
    return RB2_OK;
}

// Inner-node order of the Compact2 buffer: the reference's DFS order, or
// breadth-first so the top of the tree is contiguous.
void reorder_nodes(const std::vector<uint32_t>& in, uint32_t order, std::vector<uint32_t>& out)
{
    if (order == RB2_NODE_ORDER_DFS) { out = in; return; }
    const uint32_t n_inner = (uint32_t)(in.size() / 16);
    std::vector<uint32_t> new_of(n_inner, 0), bfs;
    bfs.reserve(n_inner);
    bfs.push_back(0);
    for (size_t h = 0; h < bfs.size(); h++) {
        const uint32_t* nd = &in[(size_t)bfs[h] * 16];
        for (int k = 0; k < 2; k++) {
            int32_t c = (int32_t)nd[12 + k];
            if (c >= 0) bfs.push_back((uint32_t)c / 4);
        }
    }
    for (uint32_t i = 0; i < (uint32_t)bfs.size(); i++) new_of[bfs[i]] = i;
    out.assign(in.size(), 0u);
    for (uint32_t i = 0; i < (uint32_t)bfs.size(); i++) {
        std::memcpy(&out[(size_t)i * 16], &in[(size_t)bfs[i] * 16], 64);
        for (int k = 0; k < 2; k++) {
            int32_t c = (int32_t)out[(size_t)i * 16 + 12 + k];
            if (c >= 0) out[(size_t)i * 16 + 12 + k] = new_of[(uint32_t)c / 4] * 4;
        }
    }
}

// Collapses a binary Compact2 node buffer (16 words per node, child = node
// index * 4 or ~Woop offset) into the 4-wide layout of rb2_traverse.cuh:
// starting from a node's two children, the inner entry with the largest box
// surface area is replaced by its two children until four entries are held
// or none is inner.  Child boxes keep their exact values, so every child test
// is the binary test of the same box.  Nodes are emitted breadth-first;
// `depth` returns the deepest wide level.
void collapse_wide4(const std::vector<uint32_t>& bin, std::vector<uint32_t>& wide, uint32_t& depth)
{
    struct Entry {
        int32_t child;
        float lo[3], hi[3];
    };
    auto entry_of = [&](uint32_t node, int k) {
        const uint32_t* w = &bin[(size_t)node * 16];
        Entry e;
        e.child = (int32_t)w[12 + k];
        const int xo = k ? 4 : 0, zo = k ? 10 : 8;
        e.lo[0] = u2f(w[xo + 0]); e.hi[0] = u2f(w[xo + 1]);
        e.lo[1] = u2f(w[xo + 2]); e.hi[1] = u2f(w[xo + 3]);
        e.lo[2] = u2f(w[zo + 0]); e.hi[2] = u2f(w[zo + 1]);
        return e;
    };
    auto area = [](const Entry& e) {
        const float dx = e.hi[0] - e.lo[0], dy = e.hi[1] - e.lo[1], dz = e.hi[2] - e.lo[2];
        return dx * dy + dy * dz + dz * dx;
    };
    wide.clear();
    std::vector<uint32_t> queue{0}, level{0};
    depth = 0;
    for (size_t h = 0; h < queue.size(); h++) {
        std::vector<Entry> es = {entry_of(queue[h], 0), entry_of(queue[h], 1)};
        while (es.size() < 4) {
            int best = -1;
            float best_a = -1.0f;
            for (int i = 0; i < (int)es.size(); i++)
                if (es[i].child >= 0 && area(es[i]) > best_a) { best = i; best_a = area(es[i]); }
            if (best < 0) break;
            const uint32_t node = (uint32_t)es[best].child / 4;
            es[best] = entry_of(node, 0);
            es.insert(es.begin() + best + 1, entry_of(node, 1));
        }
        depth = std::max(depth, level[h] + 1);
        const size_t base = wide.size();
        wide.resize(base + 32, 0u);
        for (int i = 0; i < 4; i++) {
            uint32_t child = (uint32_t)rb2dev::kWideEmpty;
            if (i < (int)es.size()) {
                const Entry& e = es[i];
                wide[base + 0 + i] = f2u(e.lo[0]); wide[base + 4 + i] = f2u(e.hi[0]);
                wide[base + 8 + i] = f2u(e.lo[1]); wide[base + 12 + i] = f2u(e.hi[1]);
                wide[base + 16 + i] = f2u(e.lo[2]); wide[base + 20 + i] = f2u(e.hi[2]);
                if (e.child >= 0) {
                    child = (uint32_t)(queue.size() * 8);  // float4 offset of the wide node
                    queue.push_back((uint32_t)e.child / 4);
                    level.push_back(level[h] + 1);
                } else {
                    child = (uint32_t)e.child;
                }
            }
            wide[base + 24 + i] = child;
        }
    }
}

}  // namespace

struct rb2_tracer {
    int device = 0;
    Occupancy occ;
    float4* d_nodes = nullptr;
    float4* d_woop = nullptr;
    uint32_t* d_triidx = nullptr;
    uint64_t n_nodes_u4 = 0, n_woop_u4 = 0;
    std::vector<uint32_t> host_nodes;  // DFS order, kept for re-layout
    uint32_t node_order = RB2_NODE_ORDER_DFS;   // layout the bulk traversals use
    uint32_t binary_order = RB2_NODE_ORDER_DFS; // order held by d_nodes (integrators use it)
    float4* d_wide = nullptr;                   // 4-wide layout, built on first use
    uint64_t n_wide_u4 = 0;
    float4* d_cw_nodes = nullptr;               // compressed 8-wide layout, built on first use
    float4* d_cw_woop = nullptr;
    uint32_t* d_cw_triidx = nullptr;            // per Woop row, as d_triidx
    unsigned long long* d_counters = nullptr;  // kSlots queue heads
    unsigned int* d_status = nullptr;
    uint32_t slot = 0;
    rb2_launch_config cfg{};
    // scratch for the host-buffer path
    float4* d_rays = nullptr;
    int4* d_hits = nullptr;
    uint8_t* d_mask = nullptr;
    uint64_t scratch_cap = 0;
    uint64_t device_bytes = 0;
    // Ray origins up to this distance per axis keep the compressed 8-wide
    // traversal conservative: 128 x the scene's largest coordinate (its boxes'
    // margin covers slab rounding of about |origin| x 2^-24).
    float cw8_origin_bound = 3.402823466e+38f;
    std::mutex mu;

    unsigned long long* next_counter()
    {
        std::lock_guard<std::mutex> g(mu);
        return d_counters + (slot++ % kSlots);
    }
};

namespace {

rb2dev::JobDesc job_of(const rb2_tracer* t, const float* rays, uint64_t n, uint32_t mode, const uint8_t* mask, void* out)
{
    rb2dev::JobDesc d{};
    const bool cw = t->node_order == RB2_NODE_ORDER_CW8;
    d.nodes = t->node_order == RB2_NODE_ORDER_WIDE4 ? t->d_wide : (cw ? t->d_cw_nodes : t->d_nodes);
    d.woop = cw ? t->d_cw_woop : t->d_woop;
    d.triidx = cw ? t->d_cw_triidx : t->d_triidx;
    d.rays = reinterpret_cast<const float4*>(rays);
    d.mask = mask;
    d.out = out;
    d.n = n;
    d.mode = mode;
    return d;
}

int trace_single(rb2_tracer* t, const float* d_rays, uint64_t n, uint32_t mode, const uint8_t* d_mask, void* d_out,
                 cudaStream_t s, bool binary = false)
{
    if (n == 0) return RB2_OK;
    unsigned long long* counter = t->next_counter();
    RB2_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s), "queue reset");
    rb2dev::KernelArgs a{};
    a.jobs = nullptr;
    a.start = nullptr;
    const uint32_t order = binary ? t->binary_order : t->node_order;
    a.inline_job = job_of(t, d_rays, n, mode, d_mask, d_out);
    if (binary && t->node_order != t->binary_order) {
        a.inline_job.nodes = t->d_nodes;
        a.inline_job.woop = t->d_woop;
        a.inline_job.triidx = t->d_triidx;
    }
    a.n_jobs = 1;
    a.fetch_threshold = t->cfg.fetch_threshold ? t->cfg.fetch_threshold : 20u;
    a.node_threshold = t->cfg.node_threshold ? t->cfg.node_threshold : rb2dev::default_node_threshold(layout_of(order));
    a.chunk = 1;
    a.counter = counter;
    a.status = t->d_status;
    const uint32_t block = t->cfg.block_threads ? t->cfg.block_threads : kDefaultBlock;
    return launch_jobs(a, n, block, t->cfg.ctas_per_sm, t->cfg.regs, layout_of(order), t->occ, s);
}

bool valid_regs(uint32_t r) { return r == 0 || r == 64 || r == 48 || r == 40; }

// Builds the compressed 8-wide layout from the tracer's Compact2 buffers and
// uploads it (nodes, Woop rows, and a triangle id per Woop row so hit records
// index it as they index the binary buffer).
int upload_cw8(rb2_tracer* t)
{
    std::vector<uint32_t> woop(t->n_woop_u4 * 4), triidx(t->n_woop_u4);
    RB2_CUDA(cudaDeviceSynchronize(), "sync before re-layout");
    RB2_CUDA(cudaMemcpy(woop.data(), t->d_woop, woop.size() * 4, cudaMemcpyDeviceToHost), "Woop read");
    RB2_CUDA(cudaMemcpy(triidx.data(), t->d_triidx, triidx.size() * 4, cudaMemcpyDeviceToHost), "index read");
    Cw8Layout cw;
    int rc = collapse_cw8(t->host_nodes.data(), t->host_nodes.size() / 4, woop.data(), triidx.data(), cw);
    if (rc) return rc;
    if (cw.depth > (uint32_t)rb2dev::kStackSizeCw8)
        return fail(RB2_ENOTSUP, "tree too deep for the compressed 8-wide layout's stack");
    std::vector<uint32_t> tri3((size_t)cw.n_tris * 3 + 4, 0u);
    for (uint32_t i = 0; i < cw.n_tris; i++) tri3[(size_t)i * 3] = cw.triidx[i];
    const size_t nb = cw.nodes.size() * 4, wb = std::max<size_t>(cw.woop.size() * 4, 16), ib = tri3.size() * 4;
    float4 *dn = nullptr, *dw = nullptr;
    uint32_t* di = nullptr;
    cudaError_t e;
    if ((e = rb2::dev_malloc(&dn, nb)) != cudaSuccess || (e = rb2::dev_malloc(&dw, wb)) != cudaSuccess ||
        (e = rb2::dev_malloc(&di, ib)) != cudaSuccess) {
        rb2::dev_free(dn); rb2::dev_free(dw); rb2::dev_free(di);
        return fail(RB2_ENOMEM, std::string("compressed 8-wide layout: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpy(dn, cw.nodes.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dw, cw.woop.data(), cw.woop.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(di, tri3.data(), ib, cudaMemcpyHostToDevice)) != cudaSuccess) {
        rb2::dev_free(dn); rb2::dev_free(dw); rb2::dev_free(di);
        return cuda_fail(e, "compressed 8-wide upload");
    }
    t->d_cw_nodes = dn;
    t->d_cw_woop = dw;
    t->d_cw_triidx = di;
    t->device_bytes += nb + wb + ib;
    return RB2_OK;
}

}  // namespace

extern "C" {

int rb2_tracer_create(const rb2_host_bvh* bvh, rb2_tracer** out)
{
    rb2::Range nvtx_range("rb2_tracer_create");
    if (!bvh || !out) return fail(RB2_EINVAL, "null argument");
    *out = nullptr;
    const HostBvh& h = host_of(bvh);
    uint32_t depth = 0;
    int rc = validate_compact2(h.nodes.data(), h.nodes.size() / 4, h.woop.data(), h.woop.size() / 4, h.triidx.data(),
                               h.triidx.size(), 0, &depth);
    if (rc) return rc;
    std::unique_ptr<rb2_tracer> t(new rb2_tracer());
    RB2_CUDA(cudaGetDevice(&t->device), "cudaGetDevice");
    rc = occupancy(t->occ);
    if (rc) return rc;
    t->n_nodes_u4 = h.nodes.size() / 4;
    t->n_woop_u4 = h.woop.size() / 4;
    t->host_nodes = h.nodes;
    {
        float m = 0.0f;
        for (int k = 0; k < 12 && (size_t)k < h.nodes.size(); k++) m = std::max(m, std::fabs(u2f(h.nodes[k])));
        t->cw8_origin_bound = 128.0f * std::max(m, 1e-30f);
    }
    // Two spare uint4 after the Woop buffer: the kernel fetches a triangle's
    // three rows before testing the first for the terminator.
    const size_t nb = h.nodes.size() * 4, wb = (h.woop.size() + 8) * 4, ib = h.triidx.size() * 4 + 16;
    auto cleanup = [&]() {
        rb2::dev_free(t->d_nodes); rb2::dev_free(t->d_woop); rb2::dev_free(t->d_triidx); rb2::dev_free(t->d_counters); rb2::dev_free(t->d_status);
    };
    cudaError_t e;
    if ((e = rb2::dev_malloc(&t->d_nodes, nb)) != cudaSuccess || (e = rb2::dev_malloc(&t->d_woop, wb)) != cudaSuccess ||
        (e = rb2::dev_malloc(&t->d_triidx, ib)) != cudaSuccess ||
        (e = rb2::dev_malloc(&t->d_counters, kSlots * sizeof(unsigned long long))) != cudaSuccess ||
        (e = rb2::dev_malloc(&t->d_status, sizeof(unsigned int))) != cudaSuccess) {
        cleanup();
        return fail(RB2_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpy(t->d_nodes, h.nodes.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_woop, 0, wb)) != cudaSuccess ||
        (e = cudaMemcpy(t->d_woop, h.woop.data(), h.woop.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_triidx, 0, ib)) != cudaSuccess ||
        (e = cudaMemcpy(t->d_triidx, h.triidx.data(), h.triidx.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(t->d_counters, 0, kSlots * sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMemset(t->d_status, 0, sizeof(unsigned int))) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "BVH upload");
    }
    t->device_bytes = nb + wb + ib + kSlots * sizeof(unsigned long long) + sizeof(unsigned int);
    *out = t.release();
    return RB2_OK;
}

int rb2_tracer_destroy(rb2_tracer* t)
{
    if (!t) return RB2_OK;
    rb2::dev_free(t->d_nodes);
    rb2::dev_free(t->d_woop);
    rb2::dev_free(t->d_triidx);
    rb2::dev_free(t->d_counters);
    rb2::dev_free(t->d_status);
    rb2::dev_free(t->d_rays);
    rb2::dev_free(t->d_hits);
    rb2::dev_free(t->d_mask);
    rb2::dev_free(t->d_wide);
    rb2::dev_free(t->d_cw_nodes);
    rb2::dev_free(t->d_cw_woop);
    rb2::dev_free(t->d_cw_triidx);
    delete t;
    return RB2_OK;
}

int rb2_tracer_set_launch(rb2_tracer* t, const rb2_launch_config* cfg)
{
    if (!t || !cfg) return fail(RB2_EINVAL, "null argument");
    if (cfg->block_threads && cfg->block_threads != 64 && cfg->block_threads != 128 && cfg->block_threads != 256)
        return fail(RB2_ENOTSUP, "block_threads must be 64, 128 or 256");
    if (cfg->fetch_threshold > 32) return fail(RB2_EINVAL, "fetch_threshold must be <= 32");
    if (cfg->node_threshold > 32) return fail(RB2_EINVAL, "node_threshold must be <= 32");
    if (!valid_regs(cfg->regs)) return fail(RB2_ENOTSUP, "regs must be 64, 48 or 40");
    t->cfg = *cfg;
    return RB2_OK;
}

int rb2_tracer_set_node_order(rb2_tracer* t, uint32_t order)
{
    if (!t) return fail(RB2_EINVAL, "null argument");
    if (order > RB2_NODE_ORDER_CW8) return fail(RB2_EINVAL, "unknown node order");
    if (order == t->node_order) return RB2_OK;
    if (order == RB2_NODE_ORDER_CW8) {
        if (!t->d_cw_nodes) {
            int rc = upload_cw8(t);
            if (rc) return rc;
        }
        t->node_order = order;
        return RB2_OK;
    }
    if (order == RB2_NODE_ORDER_WIDE4) {
        if (!t->d_wide) {
            std::vector<uint32_t> wide;
            uint32_t depth = 0;
            collapse_wide4(t->host_nodes, wide, depth);
            // Each wide level pushes at most three entries.
            if (3u * depth + 2u > (uint32_t)rb2dev::kStackSizeWide)
                return fail(RB2_ENOTSUP, "tree too deep for the 4-wide layout's stack");
            float4* d = nullptr;
            RB2_CUDA(rb2::dev_malloc(&d, wide.size() * 4), "wide node allocation");
            if (cudaMemcpy(d, wide.data(), wide.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
                rb2::dev_free(d);
                return fail(RB2_ECUDA, "wide node upload");
            }
            t->d_wide = d;
            t->n_wide_u4 = wide.size() / 4;
            t->device_bytes += wide.size() * 4;
        }
        t->node_order = order;
        return RB2_OK;
    }
    if (order != t->binary_order) {
        std::vector<uint32_t> nodes;
        reorder_nodes(t->host_nodes, order, nodes);
        RB2_CUDA(cudaDeviceSynchronize(), "sync before re-layout");
        RB2_CUDA(cudaMemcpy(t->d_nodes, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice), "node upload");
        t->binary_order = order;
    }
    t->node_order = order;
    return RB2_OK;
}

int rb2_tracer_get_node_order(const rb2_tracer* t, uint32_t* order)
{
    if (!t || !order) return fail(RB2_EINVAL, "null argument");
    *order = t->node_order;
    return RB2_OK;
}

int rb2_tracer_device_bytes(const rb2_tracer* t, uint64_t* bytes)
{
    if (!t || !bytes) return fail(RB2_EINVAL, "null argument");
    *bytes = t->device_bytes;
    return RB2_OK;
}

int rb2_trace(rb2_tracer* t, const float* d_rays, uint32_t n, int any_hit, const uint8_t* d_mask, rb2_hit* d_hits,
              void* stream)
{
    rb2::Range nvtx_range("rb2_trace");
    if (!t || (n && (!d_rays || !d_hits))) return fail(RB2_EINVAL, "null argument");
    if (((uintptr_t)d_rays | (uintptr_t)d_hits) & 15u) return fail(RB2_EINVAL, "rays and hits must be 16-byte aligned");
    return trace_single(t, d_rays, n, any_hit ? rb2dev::kAny : rb2dev::kClosest, d_mask, d_hits, (cudaStream_t)stream);
}

int rb2_trace_occlusion(rb2_tracer* t, const float* d_rays, uint32_t n, const uint8_t* d_mask, uint8_t* d_occluded,
                        void* stream)
{
    rb2::Range nvtx_range("rb2_trace_occlusion");
    if (!t || (n && (!d_rays || !d_occluded))) return fail(RB2_EINVAL, "null argument");
    if ((uintptr_t)d_rays & 15u) return fail(RB2_EINVAL, "rays must be 16-byte aligned");
    return trace_single(t, d_rays, n, rb2dev::kOcclusion, d_mask, d_occluded, (cudaStream_t)stream);
}

int rb2_trace_host(rb2_tracer* t, const float* h_rays, uint32_t n, int any_hit, const uint8_t* h_mask, rb2_hit* h_hits,
                   void* stream)
{
    rb2::Range nvtx_range("rb2_trace_host");
    if (!t || (n && (!h_rays || !h_hits))) return fail(RB2_EINVAL, "null argument");
    if (n == 0) return RB2_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_lock<std::mutex> g(t->mu);
    if (n > t->scratch_cap) {
        RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
        rb2::dev_free(t->d_rays); rb2::dev_free(t->d_hits); rb2::dev_free(t->d_mask);
        t->d_rays = nullptr; t->d_hits = nullptr; t->d_mask = nullptr;
        t->scratch_cap = 0;
        cudaError_t e;
        if ((e = rb2::dev_malloc(&t->d_rays, (size_t)n * 32)) != cudaSuccess ||
            (e = rb2::dev_malloc(&t->d_hits, (size_t)n * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&t->d_mask, (size_t)n)) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("scratch allocation: ") + cudaGetErrorString(e));
        t->scratch_cap = n;
    }
    RB2_CUDA(cudaMemcpyAsync(t->d_rays, h_rays, (size_t)n * 32, cudaMemcpyHostToDevice, s), "ray upload");
    if (h_mask) RB2_CUDA(cudaMemcpyAsync(t->d_mask, h_mask, n, cudaMemcpyHostToDevice, s), "mask upload");
    // trace_single takes the tracer mutex for the counter slot; release ours first.
    g.unlock();
    int rc = trace_single(t, reinterpret_cast<const float*>(t->d_rays), n, any_hit ? rb2dev::kAny : rb2dev::kClosest,
                          h_mask ? t->d_mask : nullptr, t->d_hits, s);
    if (rc) return rc;
    RB2_CUDA(cudaMemcpyAsync(h_hits, t->d_hits, (size_t)n * 16, cudaMemcpyDeviceToHost, s), "hit download");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    return RB2_OK;
}

int rb2_tracer_status(rb2_tracer* t, uint32_t* status, void* stream)
{
    if (!t || !status) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    RB2_CUDA(cudaMemcpyAsync(status, t->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "status read");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    return RB2_OK;
}

// ------------------------------------------------------------------------ batching
}  // extern "C"

struct rb2_batch {
    std::vector<rb2_trace_job> jobs;
    std::vector<rb2_tracer*> tracers;
    rb2dev::JobDesc* d_jobs = nullptr;
    unsigned long long* d_start = nullptr;
    std::vector<rb2_tracer*> unique_tracers;
    unsigned long long* d_counter = nullptr;
    unsigned int* d_status = nullptr;
    uint64_t total = 0;
    rb2_batch_config cfg{};
    Occupancy occ;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // ray reordering (cfg.reorder), allocated when first enabled: per-job
    // scene boxes, the tile table and first tile of each job, per-tile
    // counters, per-job bucket totals, scan scratch, each ray's key, the
    // (key, slot) pairs between the two passes of a wide key, the visiting order
    float4* d_boxes = nullptr;
    rb2::ReorderTile* d_tiles = nullptr;
    uint32_t* d_job_tile0 = nullptr;
    uint32_t* d_cnt = nullptr;
    uint32_t* d_tot = nullptr;
    uint32_t* d_chunk_sums = nullptr;
    uint32_t* d_keys = nullptr;
    uint2* d_pairs = nullptr;
    uint32_t* d_perm = nullptr;
    uint32_t n_tiles = 0;
    uint64_t cnt_cap = 0, tot_cap = 0, chunk_cap = 0;

    void drop_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

namespace {

int batch_enqueue(rb2_batch* b, cudaStream_t s)
{
    RB2_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s), "queue reset");
    rb2dev::KernelArgs a{};
    if (b->cfg.reorder) {
        rb2::ReorderArgs r{};
        r.jobs = b->d_jobs;
        r.start = b->d_start;
        r.boxes = b->d_boxes;
        r.n_jobs = (uint32_t)b->jobs.size();
        r.bits = b->cfg.reorder;
        r.total = b->total;
        r.tiles = b->d_tiles;
        r.job_tile0 = b->d_job_tile0;
        r.cnt = b->d_cnt;
        r.tot = b->d_tot;
        r.chunk_sums = b->d_chunk_sums;
        r.keys = b->d_keys;
        r.pairs = b->d_pairs;
        r.perm = b->d_perm;
        r.n_tiles = b->n_tiles;
        RB2_CUDA(rb2::reorder_enqueue(r, s), "ray reordering");
        a.perm = b->d_perm;
    }
    a.jobs = b->d_jobs;
    a.start = b->d_start;
    a.n_jobs = (uint32_t)b->jobs.size();
    a.fetch_threshold = b->cfg.fetch_threshold ? b->cfg.fetch_threshold : 20u;
    a.node_threshold =
        b->cfg.node_threshold ? b->cfg.node_threshold : rb2dev::default_node_threshold(layout_of(b->cfg.node_order));
    a.chunk = b->cfg.chunk ? b->cfg.chunk : 1u;
    a.counter = b->d_counter;
    a.status = b->d_status;
    return launch_jobs(a, b->total, b->cfg.block_threads ? b->cfg.block_threads : kDefaultBlock, b->cfg.ctas_per_sm,
                       b->cfg.regs, layout_of(b->cfg.node_order), b->occ, s);
}

// The job table points at each tracer's current layout; a tracer shared
// with another batch may have been switched since.
int batch_check_layout(const rb2_batch* b)
{
    for (const rb2_tracer* t : b->unique_tracers)
        if (layout_of(t->node_order) != layout_of(b->cfg.node_order))
            return fail(RB2_EINVAL, "a tracer's node layout changed since rb2_batch_set_config; set it again");
    return RB2_OK;
}

// (Re)allocates *p for at least `n` entries when its capacity `cap` is smaller.
template <typename T>
cudaError_t grow(T** p, uint64_t& cap, uint64_t n)
{
    if (n <= cap && *p) return cudaSuccess;
    rb2::dev_free(*p);
    *p = nullptr;
    cap = 0;
    const cudaError_t e = rb2::dev_malloc(p, sizeof(T) * std::max<uint64_t>(n, 1));
    if (e == cudaSuccess) cap = n;
    return e;
}

// Whether the sort's counters at `bits` per axis stay proportionate to the
// batch: (tiles + jobs) x buckets counters, at most two per ray plus 16M.  A
// batch of many tiny jobs would need far more counters than it has rays (and
// gains nothing from sorting a few rays per job).
bool reorder_fits(const rb2_batch* b, uint32_t bits)
{
    const uint64_t per = rb2::reorder_tile_rays(b->total, b->occ.sms);
    uint64_t tiles = 0;
    for (const rb2_trace_job& j : b->jobs) tiles += (j.n + per - 1) / per;
    const uint64_t counters = (tiles + b->jobs.size()) * (uint64_t)rb2::reorder_max_buckets(bits);
    return counters <= 2 * b->total + (16ull << 20);
}

// Buffers of ray reordering at `bits` per axis: each job's scene box (the union
// of the root's child boxes) as lo and 1 / extent, the tile table, counters,
// totals, scan scratch, keys, pairs (two-pass widths) and the visiting order.
int batch_prepare_reorder(rb2_batch* b, uint32_t bits)
{
    if (bits == 0) return RB2_OK;
    if (bits < rb2::kReorderMinBits || bits > rb2::kReorderMaxBits)
        return fail(RB2_EINVAL, "reorder must be 0 or 3..6 bits per axis");
    if (b->total >= 0xFFFFFFFFull) return fail(RB2_EINVAL, "ray reordering needs fewer than 2^32 rays per batch");
    if (!reorder_fits(b, bits))
        return fail(RB2_ENOTSUP, "ray reordering at " + std::to_string(bits) +
                                     " bits per axis needs more bucket counters than this batch has rays "
                                     "(many small jobs); use fewer bits or none");
    const uint32_t n = (uint32_t)b->jobs.size();
    RB2_CUDA(rb2::reorder_init(), "reordering shared memory");
    cudaError_t e = cudaSuccess;
    if (!b->d_boxes) {
        std::vector<float4> boxes(2 * (size_t)std::max<uint32_t>(n, 1));
        for (uint32_t i = 0; i < n; i++) {
            const std::vector<uint32_t>& h = b->jobs[i].tracer->host_nodes;
            float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            if (h.size() >= 12) {
                // Compact2 root: child 0's box in words 0-3 (x, y) and 8-9 (z), child 1's in 4-7 and 10-11.
                const int lo_w[2][3] = {{0, 2, 8}, {4, 6, 10}}, hi_w[2][3] = {{1, 3, 9}, {5, 7, 11}};
                for (int a = 0; a < 3; a++) {
                    lo[a] = std::min(u2f(h[lo_w[0][a]]), u2f(h[lo_w[1][a]]));
                    hi[a] = std::max(u2f(h[hi_w[0][a]]), u2f(h[hi_w[1][a]]));
                }
            }
            float sc[3];
            for (int a = 0; a < 3; a++) sc[a] = 1.0f / std::max(hi[a] - lo[a], 1e-30f);
            boxes[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
            boxes[2 * i + 1] = make_float4(sc[0], sc[1], sc[2], 0.0f);
        }
        if ((e = rb2::dev_malloc(&b->d_boxes, sizeof(float4) * boxes.size())) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("reordering boxes: ") + cudaGetErrorString(e));
        RB2_CUDA(cudaMemcpy(b->d_boxes, boxes.data(), sizeof(float4) * boxes.size(), cudaMemcpyHostToDevice),
                 "reordering boxes");
    }
    if (!b->d_tiles) {
        // Tiles of at most reorder_tile_rays() rays that never cross a job.
        const uint32_t per = rb2::reorder_tile_rays(b->total, b->occ.sms);
        std::vector<rb2::ReorderTile> tiles;
        std::vector<uint32_t> tile0(n + 1, 0);
        uint64_t at = 0;
        for (uint32_t i = 0; i < n; i++) {
            tile0[i] = (uint32_t)tiles.size();
            const uint64_t end = at + b->jobs[i].n;
            for (uint64_t t = at; t < end; t += per)
                tiles.push_back(rb2::ReorderTile{i, (uint32_t)t, (uint32_t)std::min<uint64_t>(end, t + per), 0u});
            at = end;
        }
        tile0[n] = (uint32_t)tiles.size();
        if ((e = rb2::dev_malloc(&b->d_job_tile0, sizeof(uint32_t) * (n + 1))) != cudaSuccess)
            return fail(RB2_ENOMEM, std::string("reordering tiles: ") + cudaGetErrorString(e));
        if ((e = rb2::dev_malloc(&b->d_tiles, sizeof(rb2::ReorderTile) * std::max<size_t>(tiles.size(), 1))) !=
            cudaSuccess)
            return fail(RB2_ENOMEM, std::string("reordering tiles: ") + cudaGetErrorString(e));
        if (!tiles.empty())
            RB2_CUDA(cudaMemcpy(b->d_tiles, tiles.data(), sizeof(rb2::ReorderTile) * tiles.size(),
                                cudaMemcpyHostToDevice), "reordering tiles");
        RB2_CUDA(cudaMemcpy(b->d_job_tile0, tile0.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice),
                 "reordering tiles");
        b->n_tiles = (uint32_t)tiles.size();
    }
    const uint64_t nb = rb2::reorder_max_buckets(bits), tot = (uint64_t)n * nb;
    uint64_t perm_cap = b->d_perm ? b->total : 0, keys_cap = b->d_keys ? b->total : 0;
    uint64_t pairs_cap = b->d_pairs ? b->total : 0;
    if ((e = grow(&b->d_cnt, b->cnt_cap, (uint64_t)b->n_tiles * nb)) != cudaSuccess ||
        (e = grow(&b->d_tot, b->tot_cap, tot)) != cudaSuccess ||
        (e = grow(&b->d_chunk_sums, b->chunk_cap, rb2::reorder_chunks(tot))) != cudaSuccess ||
        (e = grow(&b->d_keys, keys_cap, b->total)) != cudaSuccess ||
        (e = grow(&b->d_perm, perm_cap, b->total)) != cudaSuccess ||
        (bits > rb2::kReorderOnePassMaxBits && (e = grow(&b->d_pairs, pairs_cap, b->total)) != cudaSuccess))
        return fail(RB2_ENOMEM, std::string("ray reordering buffers: ") + cudaGetErrorString(e));
    return RB2_OK;
}

int batch_upload_jobs(rb2_batch* b)
{
    const uint32_t n = (uint32_t)b->jobs.size();
    if (n == 0) return RB2_OK;
    std::vector<rb2dev::JobDesc> descs(n);
    for (uint32_t i = 0; i < n; i++) {
        const rb2_trace_job& j = b->jobs[i];
        descs[i] = job_of(j.tracer, j.d_rays, j.n, j.mode, j.d_mask, j.d_out);
    }
    RB2_CUDA(cudaDeviceSynchronize(), "sync before job upload");
    RB2_CUDA(cudaMemcpy(b->d_jobs, descs.data(), sizeof(rb2dev::JobDesc) * n, cudaMemcpyHostToDevice), "job upload");
    return RB2_OK;
}

}  // namespace

extern "C" {

int rb2_batch_create(const rb2_trace_job* jobs, uint32_t n_jobs, rb2_batch** out)
{
    if (!out || (n_jobs && !jobs)) return fail(RB2_EINVAL, "null argument");
    if (n_jobs > rb2dev::kJobMask + 1u) return fail(RB2_EINVAL, "at most 2^30 jobs per batch");
    *out = nullptr;
    std::unique_ptr<rb2_batch> b(new rb2_batch());
    std::vector<rb2dev::JobDesc> descs(n_jobs);
    std::vector<unsigned long long> start(n_jobs + 1, 0);
    for (uint32_t i = 0; i < n_jobs; i++) {
        const rb2_trace_job& j = jobs[i];
        if (!j.tracer || (j.n && (!j.d_rays || !j.d_out))) return fail(RB2_EINVAL, "job with null tracer or buffer");
        if (j.mode > RB2_MODE_OCCLUSION) return fail(RB2_EINVAL, "unknown job mode");
        if (j.n > rb2dev::kMaxJobRays) return fail(RB2_EINVAL, "a job holds at most 2^32 - 1 rays");
        if ((uintptr_t)j.d_rays & 15u) return fail(RB2_EINVAL, "job rays must be 16-byte aligned");
        if (j.mode != RB2_MODE_OCCLUSION && ((uintptr_t)j.d_out & 15u)) return fail(RB2_EINVAL, "job hits must be 16-byte aligned");
        descs[i] = job_of(j.tracer, j.d_rays, j.n, j.mode, j.d_mask, j.d_out);
        start[i + 1] = start[i] + j.n;
    }
    b->jobs.assign(jobs, jobs + n_jobs);
    for (const auto& j : b->jobs)
        if (std::find(b->unique_tracers.begin(), b->unique_tracers.end(), j.tracer) == b->unique_tracers.end())
            b->unique_tracers.push_back(j.tracer);
    b->total = start[n_jobs];
    // The batch starts in the layout its tracers share (binary DFS when they differ).
    const uint32_t first = b->unique_tracers.empty() ? RB2_NODE_ORDER_DFS : b->unique_tracers[0]->node_order;
    bool same = true;
    for (const rb2_tracer* t : b->unique_tracers) same &= t->node_order == first;
    b->cfg.node_order = same ? first : RB2_NODE_ORDER_DFS;
    if (!same) {
        for (rb2_tracer* t : b->unique_tracers) {
            int rc2 = rb2_tracer_set_node_order(t, RB2_NODE_ORDER_DFS);
            if (rc2) return rc2;
        }
        for (uint32_t i = 0; i < n_jobs; i++)
            descs[i] = job_of(jobs[i].tracer, jobs[i].d_rays, jobs[i].n, jobs[i].mode, jobs[i].d_mask, jobs[i].d_out);
    }
    int rc = occupancy(b->occ);
    if (rc) return rc;
    cudaError_t e;
    if ((e = rb2::dev_malloc(&b->d_jobs, sizeof(rb2dev::JobDesc) * std::max<uint32_t>(1, n_jobs))) != cudaSuccess ||
        (e = rb2::dev_malloc(&b->d_start, sizeof(unsigned long long) * (n_jobs + 1))) != cudaSuccess ||
        (e = rb2::dev_malloc(&b->d_counter, sizeof(unsigned long long))) != cudaSuccess ||
        (e = rb2::dev_malloc(&b->d_status, sizeof(unsigned int))) != cudaSuccess) {
        rb2::dev_free(b->d_jobs); rb2::dev_free(b->d_start); rb2::dev_free(b->d_counter); rb2::dev_free(b->d_status);
        return fail(RB2_ENOMEM, std::string("batch allocation: ") + cudaGetErrorString(e));
    }
    if (n_jobs) RB2_CUDA(cudaMemcpy(b->d_jobs, descs.data(), sizeof(rb2dev::JobDesc) * n_jobs, cudaMemcpyHostToDevice), "job upload");
    RB2_CUDA(cudaMemcpy(b->d_start, start.data(), sizeof(unsigned long long) * (n_jobs + 1), cudaMemcpyHostToDevice), "job upload");
    RB2_CUDA(cudaMemset(b->d_status, 0, sizeof(unsigned int)), "status reset");
    *out = b.release();
    return RB2_OK;
}

int rb2_batch_destroy(rb2_batch* b)
{
    if (!b) return RB2_OK;
    b->drop_graph();
    rb2::dev_free(b->d_jobs);
    rb2::dev_free(b->d_start);
    rb2::dev_free(b->d_counter);
    rb2::dev_free(b->d_status);
    rb2::dev_free(b->d_boxes);
    rb2::dev_free(b->d_tiles);
    rb2::dev_free(b->d_job_tile0);
    rb2::dev_free(b->d_cnt);
    rb2::dev_free(b->d_tot);
    rb2::dev_free(b->d_chunk_sums);
    rb2::dev_free(b->d_keys);
    rb2::dev_free(b->d_pairs);
    rb2::dev_free(b->d_perm);
    delete b;
    return RB2_OK;
}

int rb2_batch_set_config(rb2_batch* b, const rb2_batch_config* cfg)
{
    if (!b || !cfg) return fail(RB2_EINVAL, "null argument");
    if (cfg->block_threads && cfg->block_threads != 64 && cfg->block_threads != 128 && cfg->block_threads != 256)
        return fail(RB2_ENOTSUP, "block_threads must be 64, 128 or 256");
    if (cfg->fetch_threshold > 32) return fail(RB2_EINVAL, "fetch_threshold must be <= 32");
    if (cfg->node_threshold > 32) return fail(RB2_EINVAL, "node_threshold must be <= 32");
    if (cfg->node_order > RB2_NODE_ORDER_CW8) return fail(RB2_EINVAL, "unknown node order");
    if (!valid_regs(cfg->regs)) return fail(RB2_ENOTSUP, "regs must be 64, 48 or 40");
    if (int rc0 = batch_prepare_reorder(b, cfg->reorder)) return rc0;
    b->drop_graph();
    for (rb2_tracer* t : b->unique_tracers) {
        int rc = rb2_tracer_set_node_order(t, cfg->node_order);
        if (rc) return rc;
    }
    b->cfg = *cfg;
    return batch_upload_jobs(b);
}

int rb2_batch_get_config(const rb2_batch* b, rb2_batch_config* cfg)
{
    if (!b || !cfg) return fail(RB2_EINVAL, "null argument");
    *cfg = b->cfg;
    return RB2_OK;
}

int rb2_batch_capture(rb2_batch* b, void* stream)
{
    if (!b) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) return fail(RB2_EINVAL, "graph capture needs a non-default stream");
    b->drop_graph();
    RB2_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = batch_enqueue(b, s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(e, "end capture");
    b->graph = g;
    RB2_CUDA(cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
    return RB2_OK;
}

int rb2_batch_launch(rb2_batch* b, void* stream)
{
    rb2::Range nvtx_range("rb2_batch_launch");
    if (!b) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (b->total == 0) return RB2_OK;
    int rc = batch_check_layout(b);
    if (rc) return rc;
    if (b->exec) {
        RB2_CUDA(cudaGraphLaunch(b->exec, s), "graph launch");
        return RB2_OK;
    }
    return batch_enqueue(b, s);
}

int rb2_batch_status(rb2_batch* b, uint32_t* status, void* stream)
{
    if (!b || !status) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    RB2_CUDA(cudaMemcpyAsync(status, b->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "status read");
    RB2_CUDA(cudaStreamSynchronize(s), "stream sync");
    return RB2_OK;
}

// Autotuner: for each node layout (DFS, BFS, 4-wide, compressed 8-wide) a
// coordinate-descent search of its launch shape (block x register budget
// jointly, then resident CTAs per SM, then the fetch threshold); the fastest
// layout gets a second pass and the queue chunk.  Each candidate is timed
// with CUDA events (median of `reps` launches after one warm-up, cold L2) and
// the fastest kept.
int rb2_batch_autotune(rb2_batch* b, void* stream, uint32_t reps, rb2_batch_config* best_out, double* best_ms_out)
{
    rb2::Range nvtx_range("rb2_batch_autotune");
    if (!b) return fail(RB2_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (reps == 0) reps = 3;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct EventFree {
        cudaEvent_t* a;
        cudaEvent_t* b;
        ~EventFree() { if (*a) cudaEventDestroy(*a); if (*b) cudaEventDestroy(*b); }
    } event_guard{&e0, &e1};
    RB2_CUDA(cudaEventCreate(&e0), "event");
    RB2_CUDA(cudaEventCreate(&e1), "event");
    // Each timed launch starts with a cold L2 (a write of twice its size,
    // outside the timing), as a launch does after other work.
    int dev = 0, l2 = 0;
    RB2_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    RB2_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev), "L2 size");
    const size_t flush_bytes = std::max<size_t>(2 * (size_t)l2, 1 << 20);
    void* flush = nullptr;
    if (rb2::dev_malloc(&flush, flush_bytes) != cudaSuccess) flush = nullptr;  // tune warm if memory is short
    struct FlushFree {
        void* p;
        ~FlushFree() { if (p) rb2::dev_free(p); }
    } flush_guard{flush};
    auto time_cfg = [&](const rb2_batch_config& c, double& ms) -> int {
        int rc = rb2_batch_set_config(b, &c);
        if (rc) return rc;
        rc = batch_enqueue(b, s);
        if (rc) return rc;
        std::vector<float> t(reps);
        for (uint32_t r = 0; r < reps; r++) {
            if (flush) RB2_CUDA(cudaMemsetAsync(flush, (int)(r & 0xFF), flush_bytes, s), "L2 flush");
            RB2_CUDA(cudaEventRecord(e0, s), "event");
            rc = batch_enqueue(b, s);
            if (rc) return rc;
            RB2_CUDA(cudaEventRecord(e1, s), "event");
            RB2_CUDA(cudaEventSynchronize(e1), "event sync");
            RB2_CUDA(cudaEventElapsedTime(&t[r], e0, e1), "event time");
        }
        std::sort(t.begin(), t.end());
        ms = t[reps / 2];
        return RB2_OK;
    };
    const uint32_t orders[] = {RB2_NODE_ORDER_DFS, RB2_NODE_ORDER_BFS, RB2_NODE_ORDER_WIDE4, RB2_NODE_ORDER_CW8};
    const uint32_t blocks[] = {64, 128, 256};
    const uint32_t regs[] = {64, 48, 40};
    const uint32_t thresholds[] = {8, 16, 20, 24, 28};
    const uint32_t node_thresholds[] = {1, 4, 8, 12, 16, 20};
    const uint32_t chunks[] = {1, 2, 4, 8};
    // One coordinate-descent pass over the launch shape of a fixed layout:
    // block x register budget jointly, then the node-phase threshold, then
    // resident CTAs, then the fetch threshold.
    auto tune_shape = [&](rb2_batch_config& cur, double& cur_ms) -> int {
        int rc2;
        for (uint32_t bl : blocks) {
            for (uint32_t rg : regs) {
                rb2_batch_config c = cur;
                c.block_threads = bl; c.regs = rg; c.ctas_per_sm = 0;
                double ms;
                if ((rc2 = time_cfg(c, ms))) return rc2;
                if (ms < cur_ms) { cur = c; cur_ms = ms; }
            }
        }
        for (uint32_t nt : node_thresholds) {
            rb2_batch_config c = cur; c.node_threshold = nt; double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if (ms < cur_ms) { cur = c; cur_ms = ms; }
        }
        const int maxc =
            std::max(1, b->occ.per_sm[block_index(cur.block_threads)][regs_index(cur.regs)][layout_of(cur.node_order)]);
        for (int k : {maxc, std::max(1, maxc * 3 / 4), std::max(1, maxc / 2)}) {
            rb2_batch_config c = cur; c.ctas_per_sm = (uint32_t)k; double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if (ms < cur_ms) { cur = c; cur_ms = ms; }
        }
        for (uint32_t th : thresholds) {
            rb2_batch_config c = cur; c.fetch_threshold = th; double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if (ms < cur_ms) { cur = c; cur_ms = ms; }
        }
        return RB2_OK;
    };
    // The whole search at one reordering setting: each layout gets its own
    // shape search (the layouts favour different register budgets and
    // thresholds); the winner gets a second pass and the queue chunk; then a
    // last look at the layouts, each with its own tuned shape, re-timed with
    // the incumbent so drift between searches cannot decide it.
    auto search = [&](uint32_t reorder, rb2_batch_config& best, double& best_ms) -> int {
        int rc2;
        best = rb2_batch_config{};
        best.block_threads = kDefaultBlock;
        best.fetch_threshold = 20;
        best.chunk = 1;
        best.node_order = RB2_NODE_ORDER_DFS;
        best.regs = 64;
        best.reorder = reorder;
        if ((rc2 = time_cfg(best, best_ms))) return rc2;
        std::vector<rb2_batch_config> per_layout;
        for (uint32_t o : orders) {
            rb2_batch_config c = best;
            c.node_order = o;
            double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if ((rc2 = tune_shape(c, ms))) return rc2;
            per_layout.push_back(c);
            if (ms < best_ms) { best = c; best_ms = ms; }
        }
        if ((rc2 = tune_shape(best, best_ms))) return rc2;
        for (uint32_t ch : chunks) {
            rb2_batch_config c = best; c.chunk = ch; double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if (ms < best_ms) { best = c; best_ms = ms; }
        }
        double inc_ms;
        if ((rc2 = time_cfg(best, inc_ms))) return rc2;
        best_ms = inc_ms;
        for (const rb2_batch_config& c : per_layout) {
            if (c.node_order == best.node_order) continue;
            double ms;
            if ((rc2 = time_cfg(c, ms))) return rc2;
            if (ms < best_ms) { best = c; best_ms = ms; }
        }
        return RB2_OK;
    };
    rb2_batch_config best{}, best_r{};
    double best_ms = 0, best_r_ms = 0;
    int rc = search(0, best, best_ms);
    if (rc) return rc;
    // Ray reordering (when the batch's rays fit its 32-bit visiting order and
    // its sort counters stay proportionate): the search again with 4 bits per
    // axis, then the other widths on its winner.
    if (b->total < 0xFFFFFFFFull && reorder_fits(b, 4)) {
        if ((rc = search(4, best_r, best_r_ms))) return rc;
        for (uint32_t bits : {3u, 5u, 6u}) {
            if (!reorder_fits(b, bits)) continue;
            rb2_batch_config c = best_r; c.reorder = bits; double ms;
            if ((rc = time_cfg(c, ms))) return rc;
            if (ms < best_r_ms) { best_r = c; best_r_ms = ms; }
        }
        double ms0;
        if ((rc = time_cfg(best, ms0))) return rc;
        if ((rc = time_cfg(best_r, best_r_ms))) return rc;
        best_ms = ms0;
        if (best_r_ms < best_ms) { best = best_r; best_ms = best_r_ms; }
    }
    rc = rb2_batch_set_config(b, &best);
    if (rc) return rc;
    if (best_out) *best_out = best;
    if (best_ms_out) *best_ms_out = best_ms;
    return RB2_OK;
}

// ------------------------------------------------------------------ camera entry points
int rb2_camera_rays(const rb2_camera* cam, uint32_t spp, uint64_t seed, int jitter, float* d_rays, void* stream)
{
    if (!cam || !d_rays || spp == 0) return fail(RB2_EINVAL, "bad camera-ray arguments");
    rb2dev::CamArgs c;
    std::memcpy(c.r2c, cam->raster_to_camera, sizeof(c.r2c));
    std::memcpy(c.c2w, cam->camera_to_world, sizeof(c.c2w));
    c.width = cam->width; c.height = cam->height; c.spp = spp; c.jitter = jitter ? 1u : 0u; c.seed = seed;
    uint64_t total = (uint64_t)cam->width * cam->height * spp;
    unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
    rb2dev::k_camera_rays<<<std::max(1u, blocks), 256, 0, (cudaStream_t)stream>>>(c, reinterpret_cast<float4*>(d_rays));
    RB2_CUDA(cudaGetLastError(), "camera launch");
    return RB2_OK;
}

int rb2_camera_rays_at(const rb2_camera* cam, const float* d_raster_xy, uint32_t n, float* d_rays, void* stream)
{
    if (!cam || (n && (!d_raster_xy || !d_rays))) return fail(RB2_EINVAL, "bad camera-ray arguments");
    if (n == 0) return RB2_OK;
    rb2dev::CamArgs c;
    std::memcpy(c.r2c, cam->raster_to_camera, sizeof(c.r2c));
    std::memcpy(c.c2w, cam->camera_to_world, sizeof(c.c2w));
    c.width = cam->width; c.height = cam->height; c.spp = 1; c.jitter = 0; c.seed = 0;
    unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    rb2dev::k_camera_rays_at<<<std::max(1u, blocks), 256, 0, (cudaStream_t)stream>>>(
        c, reinterpret_cast<const float2*>(d_raster_xy), n, reinterpret_cast<float4*>(d_rays));
    RB2_CUDA(cudaGetLastError(), "camera launch");
    return RB2_OK;
}

}  // extern "C"

namespace rb2 {
DeviceBvhView device_bvh(const rb2_tracer* t, bool allow_cw8)
{
    if (allow_cw8 && t->node_order == RB2_NODE_ORDER_CW8)
        return DeviceBvhView{t->d_cw_nodes, t->d_cw_woop, t->d_cw_triidx, t->d_status, true};
    return DeviceBvhView{t->d_nodes, t->d_woop, t->d_triidx, t->d_status, false};
}

unsigned long long* tracer_queue_counter(rb2_tracer* t) { return t->next_counter(); }

bool cw8_origin_ok(const rb2_tracer* t, const float* o)
{
    const float b = t->cw8_origin_bound;
    return std::fabs(o[0]) <= b && std::fabs(o[1]) <= b && std::fabs(o[2]) <= b;
}

int trace_binary(rb2_tracer* t, const float* d_rays, uint64_t n, int any_hit, void* d_out, void* stream)
{
    return trace_single(t, d_rays, n, any_hit ? rb2dev::kAny : rb2dev::kClosest, nullptr, d_out,
                        (cudaStream_t)stream, true);
}
}  // namespace rb2

extern "C" int rb2_tracer_dev_bvh(const rb2_tracer* t, rb2_dev_bvh* out)
{
    if (!t || !out) return fail(RB2_EINVAL, "null argument");
    out->nodes = t->d_nodes;
    out->woop = t->d_woop;
    out->triidx = t->d_triidx;
    out->n_nodes_u4 = t->n_nodes_u4;
    out->n_woop_u4 = t->n_woop_u4;
    return RB2_OK;
}

// ------------------------------------------------------------------ pipelined host path
struct rb2_pipeline {
    struct Slot {
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        float4* d_rays = nullptr;
        int4* d_out = nullptr;
        uint8_t* d_mask = nullptr;
        bool busy = false;
    };
    std::vector<Slot> slots;
    uint64_t chunk = 0;
    cudaEvent_t entry = nullptr;  // recorded on the caller's stream at entry
};

extern "C" {

int rb2_pipeline_destroy(rb2_pipeline* p)
{
    if (!p) return RB2_OK;
    for (auto& s : p->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        rb2::dev_free(s.d_rays);
        rb2::dev_free(s.d_out);
        rb2::dev_free(s.d_mask);
        if (s.done) cudaEventDestroy(s.done);
        if (s.stream) cudaStreamDestroy(s.stream);
    }
    if (p->entry) cudaEventDestroy(p->entry);
    delete p;
    return RB2_OK;
}

int rb2_pipeline_create(uint64_t chunk_rays, uint32_t depth, rb2_pipeline** out)
{
    if (!out || chunk_rays == 0 || chunk_rays > 0xFFFFFFFFull || depth == 0 || depth > 16)
        return fail(RB2_EINVAL, "pipeline needs 0 < chunk_rays < 2^32 and 0 < depth <= 16");
    *out = nullptr;
    std::unique_ptr<rb2_pipeline> p(new rb2_pipeline());
    p->chunk = chunk_rays;
    p->slots.resize(depth);
    if (cudaEventCreateWithFlags(&p->entry, cudaEventDisableTiming) != cudaSuccess) {
        rb2_pipeline_destroy(p.release());
        return fail(RB2_ECUDA, "pipeline event");
    }
    for (auto& s : p->slots) {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = rb2::dev_malloc(&s.d_rays, chunk_rays * 32)) != cudaSuccess ||
            (e = rb2::dev_malloc(&s.d_out, chunk_rays * 16)) != cudaSuccess ||
            (e = rb2::dev_malloc(&s.d_mask, chunk_rays)) != cudaSuccess) {
            rb2_pipeline_destroy(p.release());
            return fail(RB2_ENOMEM, std::string("pipeline staging: ") + cudaGetErrorString(e));
        }
    }
    *out = p.release();
    return RB2_OK;
}

int rb2_trace_host_jobs(rb2_pipeline* p, const rb2_host_job* jobs, uint32_t n_jobs, void* stream)
{
    rb2::Range nvtx_range("rb2_trace_host_jobs");
    if (!p || (n_jobs && !jobs)) return fail(RB2_EINVAL, "null argument");
    const cudaStream_t caller = (cudaStream_t)stream;
    for (uint32_t i = 0; i < n_jobs; i++) {
        const rb2_host_job& j = jobs[i];
        if (!j.tracer || (j.n && (!j.h_rays || !j.h_out)) || j.mode > RB2_MODE_OCCLUSION)
            return fail(RB2_EINVAL, "bad host job");
    }
    const size_t nslots = p->slots.size();
    // Work ordered after what the caller queued on `stream`.
    RB2_CUDA(cudaEventRecord(p->entry, caller), "pipeline entry");
    for (auto& s : p->slots) RB2_CUDA(cudaStreamWaitEvent(s.stream, p->entry, 0), "pipeline entry wait");
    size_t k = 0;
    for (uint32_t i = 0; i < n_jobs; i++) {
        const rb2_host_job& j = jobs[i];
        const size_t out_b = j.mode == RB2_MODE_OCCLUSION ? 1 : 16;
        for (uint64_t off = 0; off < j.n; off += p->chunk, k++) {
            const uint64_t n = std::min<uint64_t>(p->chunk, j.n - off);
            auto& s = p->slots[k % nslots];
            if (s.busy) RB2_CUDA(cudaEventSynchronize(s.done), "pipeline slot wait");
            RB2_CUDA(cudaMemcpyAsync(s.d_rays, j.h_rays + 8 * off, n * 32, cudaMemcpyHostToDevice, s.stream), "chunk upload");
            if (j.h_mask) RB2_CUDA(cudaMemcpyAsync(s.d_mask, j.h_mask + off, n, cudaMemcpyHostToDevice, s.stream), "mask upload");
            const uint8_t* mask = j.h_mask ? s.d_mask : nullptr;
            int rc = j.mode == RB2_MODE_OCCLUSION
                         ? trace_single(j.tracer, reinterpret_cast<const float*>(s.d_rays), n, rb2dev::kOcclusion, mask,
                                        s.d_out, s.stream)
                         : trace_single(j.tracer, reinterpret_cast<const float*>(s.d_rays), n,
                                        j.mode == RB2_MODE_ANY ? rb2dev::kAny : rb2dev::kClosest, mask, s.d_out, s.stream);
            if (rc) return rc;
            RB2_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(j.h_out) + off * out_b, s.d_out, n * out_b,
                                     cudaMemcpyDeviceToHost, s.stream), "chunk download");
            RB2_CUDA(cudaEventRecord(s.done, s.stream), "pipeline event");
            s.busy = true;
        }
    }
    // `stream` waits for every chunk, so events recorded on it bracket the
    // whole pipelined job set (copies included).
    for (auto& s : p->slots) {
        if (!s.busy) continue;
        RB2_CUDA(cudaStreamWaitEvent(caller, s.done, 0), "pipeline join");
        RB2_CUDA(cudaEventSynchronize(s.done), "pipeline drain");
        s.busy = false;
    }
    return RB2_OK;
}

}  // extern "C"
