// C-ABI glue for the host side: errors, build, buffers, cache.
#include "rb2_internal.h"

#include <chrono>
#include <new>

struct rb2_host_bvh {
    rb2::HostBvh b;
};

namespace rb2 {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    set_error(msg);
    return code;
}

int save_binary(const HostBvh& b, const char* path);
int save_text(const HostBvh& b, const char* path);
int load_any(const char* path, HostBvh& b);

}  // namespace rb2

using namespace rb2;

extern "C" {

const char* rb2_last_error(void) { return g_last_error.c_str(); }

const char* rb2_version(void) { return "rb2 1.0 (sm_100a)"; }

int rb2_build_params_default(rb2_build_params* p)
{
    if (!p) return fail(RB2_EINVAL, "null params");
    p->sah_node_cost = 1.0f;
    p->sah_triangle_cost = 1.0f;
    p->min_leaf_size = 1;
    p->max_leaf_size = 0x7FFFFFF;
    p->split_alpha = 1.0e-5f;
    p->max_depth = 64;
    p->max_spatial_depth = 48;
    p->spatial_bins = 64;
    p->object_bins = 64;
    p->exact_sweep_max = 512;
    p->num_threads = 0;
    p->layout = RB2_LAYOUT_COMPACT2;
    return RB2_OK;
}

int rb2_bvh_build(const float* v_xyz, uint32_t nv, const uint32_t* idx3, uint32_t ntri, const rb2_build_params* params,
                  rb2_host_bvh** out)
{
    rb2::Range nvtx_range("rb2_bvh_build");
    if (!out) return fail(RB2_EINVAL, "null output handle");
    *out = nullptr;
    if ((ntri && (!v_xyz || !idx3)) || (nv && !v_xyz)) return fail(RB2_EINVAL, "null geometry");
    rb2_build_params p;
    if (params) p = *params; else rb2_build_params_default(&p);
    if (p.layout != RB2_LAYOUT_COMPACT2) return fail(RB2_ENOTSUP, "only the Compact2 layout is supported");
    if (p.max_depth == 0 || p.max_depth > 64) return fail(RB2_EINVAL, "max_depth must be in [1, 64]");
    try {
        auto t0 = std::chrono::steady_clock::now();
        std::unique_ptr<rb2_host_bvh> h(new rb2_host_bvh());
        Tree tree;
        int rc = build_tree(v_xyz, nv, idx3, ntri, p, tree, h->b.counts);
        if (rc) return rc;
        rb2_bvh_counts keep = h->b.counts;
        rc = pack_compact2(tree, v_xyz, idx3, h->b);
        if (rc) return rc;
        auto t1 = std::chrono::steady_clock::now();
        rb2_bvh_counts& c = h->b.counts;
        c.n_inner = keep.n_inner;
        c.n_leaves = keep.n_leaves;
        c.n_tri_refs = keep.n_tri_refs;
        c.n_tris = ntri;
        c.max_depth = keep.max_depth;
        c.sah = keep.sah;
        c.build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        h->b.verts.assign(v_xyz, v_xyz + 3 * (size_t)nv);
        h->b.idx.assign(idx3, idx3 + 3 * (size_t)ntri);
        *out = h.release();
        return RB2_OK;
    } catch (const std::bad_alloc&) {
        return fail(RB2_ENOMEM, "host allocation failed during build");
    }
}

int rb2_bvh_from_buffers(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop, uint64_t n_woop_u4,
                         const uint32_t* triidx, uint64_t n_triidx, rb2_host_bvh** out)
{
    if (!out) return fail(RB2_EINVAL, "null output handle");
    *out = nullptr;
    if (!nodes || !woop || !triidx) return fail(RB2_EINVAL, "null buffer");
    uint32_t depth = 0;
    int rc = validate_compact2(nodes, n_nodes_u4, woop, n_woop_u4, triidx, n_triidx, 0, &depth);
    if (rc) return rc;
    try {
        std::unique_ptr<rb2_host_bvh> h(new rb2_host_bvh());
        h->b.nodes.assign(nodes, nodes + 4 * n_nodes_u4);
        h->b.woop.assign(woop, woop + 4 * n_woop_u4);
        h->b.triidx.assign(triidx, triidx + n_triidx);
        rb2_bvh_counts& c = h->b.counts;
        c.n_nodes_u4 = n_nodes_u4;
        c.n_woop_u4 = n_woop_u4;
        c.n_triidx = n_triidx;
        c.n_inner = (uint32_t)(n_nodes_u4 / 4);
        c.max_depth = depth;
        c.layout = RB2_LAYOUT_COMPACT2;
        *out = h.release();
        return RB2_OK;
    } catch (const std::bad_alloc&) {
        return fail(RB2_ENOMEM, "host allocation failed");
    }
}

int rb2_bvh_counts_get(const rb2_host_bvh* b, rb2_bvh_counts* out)
{
    if (!b || !out) return fail(RB2_EINVAL, "null argument");
    *out = b->b.counts;
    return RB2_OK;
}

const uint32_t* rb2_bvh_nodes(const rb2_host_bvh* b) { return b ? b->b.nodes.data() : nullptr; }
const uint32_t* rb2_bvh_woop(const rb2_host_bvh* b) { return b ? b->b.woop.data() : nullptr; }
const uint32_t* rb2_bvh_triidx(const rb2_host_bvh* b) { return b ? b->b.triidx.data() : nullptr; }

void rb2_host_bvh_free(rb2_host_bvh* b) { delete b; }

int rb2_bvh_save(const rb2_host_bvh* b, const char* path)
{
    if (!b || !path) return fail(RB2_EINVAL, "null argument");
    return save_binary(b->b, path);
}

int rb2_bvh_save_text(const rb2_host_bvh* b, const char* path)
{
    if (!b || !path) return fail(RB2_EINVAL, "null argument");
    return save_text(b->b, path);
}

int rb2_bvh_load(const char* path, rb2_host_bvh** out)
{
    if (!path || !out) return fail(RB2_EINVAL, "null argument");
    *out = nullptr;
    try {
        std::unique_ptr<rb2_host_bvh> h(new rb2_host_bvh());
        int rc = load_any(path, h->b);
        if (rc) return rc;
        *out = h.release();
        return RB2_OK;
    } catch (const std::bad_alloc&) {
        return fail(RB2_ENOMEM, "host allocation failed while loading");
    }
}

}  // extern "C"

// Accessor used by the CUDA side (rb2_trace.cu) to reach the host buffers.
namespace rb2 {
const HostBvh& host_of(const rb2_host_bvh* b) { return b->b; }
}  // namespace rb2
