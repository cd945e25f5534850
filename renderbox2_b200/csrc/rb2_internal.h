// Internal helpers shared by the host-side C++ sources of librb2.
#pragma once

#include "rb2.h"
#include "rb2_render.h"

#include <nvtx3/nvToolsExt.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace rb2 {

// ---- error channel ------------------------------------------------------------
// Every C-ABI entry point returns an rb2_status; the text of the most recent
// failure on the calling thread is kept for rb2_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

// ---- small vector math (host) ---------------------------------------------------
// Definitions match the reference's helper_math usage: dot/cross left to right,
// normalize = v * (1/sqrtf(dot(v,v))).  Host sources are compiled with
// -ffp-contract=off so each operation rounds once, as written.
struct f3 {
    float x, y, z;
};
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline f3 operator*(float s, f3 a) { return mk(a.x * s, a.y * s, a.z * s); }
inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline f3 cross(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline f3 normalize(f3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
inline float get(const f3& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }
inline float& get(f3& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }

// Compare-select min/max: inlined (libm fminf/fmaxf are out-of-line calls
// without -ffinite-math-only) and equivalent for the finite coordinates of
// valid geometry.
inline float mn(float a, float b) { return b < a ? b : a; }
inline float mx(float a, float b) { return b > a ? b : a; }

struct Box {
    f3 lo{FLT_MAX, FLT_MAX, FLT_MAX};
    f3 hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    bool valid() const { return lo.x <= hi.x && lo.y <= hi.y && lo.z <= hi.z; }
    void insert(f3 p)
    {
        lo = mk(mn(lo.x, p.x), mn(lo.y, p.y), mn(lo.z, p.z));
        hi = mk(mx(hi.x, p.x), mx(hi.y, p.y), mx(hi.z, p.z));
    }
    void grow(const Box& b)
    {
        lo = mk(mn(lo.x, b.lo.x), mn(lo.y, b.lo.y), mn(lo.z, b.lo.z));
        hi = mk(mx(hi.x, b.hi.x), mx(hi.y, b.hi.y), mx(hi.z, b.hi.z));
    }
    void clip(const Box& b)
    {
        lo = mk(mx(lo.x, b.lo.x), mx(lo.y, b.lo.y), mx(lo.z, b.lo.z));
        hi = mk(mn(hi.x, b.hi.x), mn(hi.y, b.hi.y), mn(hi.z, b.hi.z));
    }
    float area() const
    {
        if (!valid()) return 0.0f;
        f3 d = hi - lo;
        return (d.x * d.y + d.y * d.z + d.z * d.x) * 2.0f;
    }
};

// ---- host BVH object (what rb2_host_bvh points to) -------------------------------
struct HostBvh {
    uint32_t layout = RB2_LAYOUT_COMPACT2;
    std::vector<uint32_t> nodes;   // 4 words per uint4
    std::vector<uint32_t> woop;    // 4 words per uint4
    std::vector<uint32_t> triidx;  // one per woop uint4 slot
    rb2_bvh_counts counts{};
    // Scene geometry kept for integrators (optional; empty when loaded from a cache).
    std::vector<float> verts;      // xyz per vertex
    std::vector<uint32_t> idx;     // 3 per triangle
};

// Binary tree produced by the builder, consumed by the packer.
struct TreeNode {
    Box box;
    int32_t child[2] = {-1, -1};   // indices into Tree::nodes; -1 for leaves
    uint32_t tri_begin = 0, tri_count = 0;  // range in Tree::tri_refs (leaves)
    bool leaf() const { return child[0] < 0; }
};
struct Tree {
    std::vector<TreeNode> nodes;   // nodes[0] is the root
    std::vector<uint32_t> tri_refs;
};

// Packs a binary tree into the Compact2 layout.  Node slot order, child index
// encoding and the Woop transform follow the reference packer
// (accelerators/sbvh/cudabvh.cpp:216-322) so reference-built and rb2-built
// buffers are interchangeable.
int pack_compact2(const Tree& tree, const float* v, const uint32_t* idx, HostBvh& out);

// Woop coefficients of one triangle: 12 words, rows (w0, w1, w2).
void woopify(const f3& v0, const f3& v1, const f3& v2, uint32_t out12[12]);

int build_tree(const float* v, uint32_t nv, const uint32_t* idx, uint32_t ntri, const rb2_build_params& p,
               Tree& tree, rb2_bvh_counts& counts);

// Validates a Compact2 buffer set: every child index in range, every leaf run
// terminated, the node graph a tree of bounded depth.  Used before upload so a
// traversal kernel can never loop or read out of bounds.
int validate_compact2(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop, uint64_t n_woop_u4,
                      const uint32_t* triidx, uint64_t n_triidx, uint32_t n_tris_hint, uint32_t* max_depth_out);

// Compressed 8-wide layout (rb2_cw8.cpp) collapsed from a Compact2 buffer set
// that validate_compact2 accepted.
struct Cw8Layout {
    std::vector<uint32_t> nodes;   // 20 words per node
    std::vector<uint32_t> woop;    // 12 words (3 Woop rows) per triangle
    std::vector<uint32_t> triidx;  // original triangle id per triangle
    uint32_t n_nodes = 0, n_tris = 0, depth = 0;
};
int collapse_cw8(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop, const uint32_t* triidx,
                 Cw8Layout& out);

// Device view of a tracer's BVH (defined in rb2_trace.cu) for integrator
// kernels: the compressed 8-wide layout when the tracer uses it and the caller
// can traverse it (cw8 set), else the binary Compact2 buffer.
struct DeviceBvhView {
    const void* nodes;    // float4*
    const void* woop;     // float4*
    const uint32_t* triidx;
    unsigned int* status;
    bool cw8;
};
DeviceBvhView device_bvh(const rb2_tracer* t, bool allow_cw8 = false);

// Checks a film filter description (rb2_film_table.cpp).
int validate_filter(const rb2_filter* f);

// A zeroed-before-use queue head of the tracer's ring (one per launch in flight).
// The ring holds kTracerQueueSlots heads, so at most that many launches of one
// tracer may be in flight at once.
constexpr uint32_t kTracerQueueSlots = 256;
unsigned long long* tracer_queue_counter(rb2_tracer* t);

// Whether rays from origin o keep the compressed 8-wide traversal exact (its
// boxes' margin covers slab rounding for origins within 128 x the scene's
// largest coordinate); integrators trace camera rays from farther away through
// the binary buffer.
bool cw8_origin_ok(const rb2_tracer* t, const float* o);
// Bulk trace through the binary buffer whatever the tracer's node order.
int trace_binary(rb2_tracer* t, const float* d_rays, uint64_t n, int any_hit, void* d_out, void* stream);

// A named profiler range over one host-side stage of the library (NVTX, header
// only: without a profiler attached, such as `ncu --nvtx`, it costs a branch).
// Ranges nest with scope; the names are the C-ABI entry points.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

}  // namespace rb2
