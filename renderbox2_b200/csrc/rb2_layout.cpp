// Compact2 packer, Woop transform, layout validation and the BVH cache.
#include "rb2_internal.h"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>

namespace rb2 {

namespace {

// General 4x4 inverse by cofactor expansion (the MESA gluInvertMatrix
// formulation, which the reference's Matrix4x4::invert uses,
// core/transform.h:205-333).  The terms are evaluated in the same order and
// without contraction so the Woop rows are bit-identical to the reference's
// packer; m is row-major.
void invert4(const float m[16], float out[16])
{
    float inv[16];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
             m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
             m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
             m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
              m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
             m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
             m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
             m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
              m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
             m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
             m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
              m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
              m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
             m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
             m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
              m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
              m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    float det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    det = 1.0f / det;
    for (int i = 0; i < 16; i++) out[i] = inv[i] * det;
}

}  // namespace

void invert4_public(const float m[16], float out[16]) { invert4(m, out); }

// Woop's unit-triangle transform (cudabvh.cpp:303-322): columns of M are
// v0-v2, v1-v2, normalize(cross(v0-v2, v1-v2)) and the point v2; the rows of
// M^-1 give w0 = (row2.xyz, -row2.w), w1 = row0, w2 = row1.
void woopify(const f3& v0, const f3& v1, const f3& v2, uint32_t out[12])
{
    f3 e0 = v0 - v2, e1 = v1 - v2;
    f3 n = normalize(cross(e0, e1));
    float m[16] = {e0.x, e1.x, n.x, v2.x,
                   e0.y, e1.y, n.y, v2.y,
                   e0.z, e1.z, n.z, v2.z,
                   0.0f, 0.0f, 0.0f, 1.0f};
    float inv[16];
    invert4(m, inv);
    float w0x = inv[8];
    if (w0x == 0.0f) w0x = 0.0f;  // -0.0 would read as a leaf terminator (cudabvh.cpp:265-266)
    out[0] = f2u(w0x);
    out[1] = f2u(inv[9]);
    out[2] = f2u(inv[10]);
    out[3] = f2u(-inv[11]);
    for (int k = 0; k < 4; k++) out[4 + k] = f2u(inv[k]);
    for (int k = 0; k < 4; k++) out[8 + k] = f2u(inv[4 + k]);
}

// Flattening order follows create_compact (cudabvh.cpp:216-296): a LIFO stack
// of inner nodes; when a node is popped its inner children get the next two
// node slots (child index = uint4 offset, i.e. bytes/16) and its leaf children
// append their Woop triangles plus a -0.0 terminator (child index = ~offset).
int pack_compact2(const Tree& tree, const float* v, const uint32_t* idx, HostBvh& out)
{
    if (tree.nodes.empty() || tree.nodes[0].leaf()) return fail(RB2_EINVAL, "packer needs an inner root");
    const f3* V = reinterpret_cast<const f3*>(v);
    out.nodes.assign(16, 0u);
    out.woop.clear();
    out.triidx.clear();
    out.woop.reserve((size_t)(tree.tri_refs.size() * 3 + tree.nodes.size()) * 4);
    out.triidx.reserve(tree.tri_refs.size() * 3 + tree.nodes.size());
    struct Entry { int32_t node; uint32_t slot; };
    std::vector<Entry> stack;
    stack.push_back({0, 0});
    while (!stack.empty()) {
        Entry e = stack.back();
        stack.pop_back();
        const TreeNode& tn = tree.nodes[e.node];
        int32_t cidx[2];
        for (int i = 0; i < 2; i++) {
            const TreeNode& ch = tree.nodes[tn.child[i]];
            if (!ch.leaf()) {
                uint32_t slot = (uint32_t)(out.nodes.size() / 4);
                cidx[i] = (int32_t)slot;
                stack.push_back({tn.child[i], slot});
                out.nodes.resize(out.nodes.size() + 16, 0u);
                continue;
            }
            cidx[i] = ~(int32_t)(out.woop.size() / 4);
            for (uint32_t j = 0; j < ch.tri_count; j++) {
                uint32_t tri = tree.tri_refs[ch.tri_begin + j];
                uint32_t w[12];
                woopify(V[idx[3 * tri + 0]], V[idx[3 * tri + 1]], V[idx[3 * tri + 2]], w);
                out.woop.insert(out.woop.end(), w, w + 12);
                out.triidx.push_back(tri);
                out.triidx.push_back(0);
                out.triidx.push_back(0);
            }
            for (int k = 0; k < 4; k++) out.woop.push_back(0x80000000u);
            out.triidx.push_back(0);
        }
        const Box& b0 = tree.nodes[tn.child[0]].box;
        const Box& b1 = tree.nodes[tn.child[1]].box;
        uint32_t* dst = &out.nodes[(size_t)e.slot * 4];
        dst[0] = f2u(b0.lo.x); dst[1] = f2u(b0.hi.x); dst[2] = f2u(b0.lo.y); dst[3] = f2u(b0.hi.y);
        dst[4] = f2u(b1.lo.x); dst[5] = f2u(b1.hi.x); dst[6] = f2u(b1.lo.y); dst[7] = f2u(b1.hi.y);
        dst[8] = f2u(b0.lo.z); dst[9] = f2u(b0.hi.z); dst[10] = f2u(b1.lo.z); dst[11] = f2u(b1.hi.z);
        dst[12] = (uint32_t)cidx[0]; dst[13] = (uint32_t)cidx[1]; dst[14] = 0; dst[15] = 0;
    }
    out.counts.n_nodes_u4 = out.nodes.size() / 4;
    out.counts.n_woop_u4 = out.woop.size() / 4;
    out.counts.n_triidx = out.triidx.size();
    out.counts.layout = RB2_LAYOUT_COMPACT2;
    return RB2_OK;
}

int validate_compact2(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop, uint64_t n_woop_u4,
                      const uint32_t* triidx, uint64_t n_triidx, uint32_t n_tris_hint, uint32_t* max_depth_out)
{
    if (n_nodes_u4 < 4 || n_nodes_u4 % 4 != 0) return fail(RB2_EFORMAT, "node buffer must hold whole 64-byte nodes");
    if (n_nodes_u4 >= 0x76543210ull) return fail(RB2_EFORMAT, "node buffer too large for 31-bit child indices");
    if (n_woop_u4 >= 0x7fffffffull) return fail(RB2_EFORMAT, "Woop buffer too large");
    if (n_triidx != n_woop_u4) return fail(RB2_EFORMAT, "triangle index buffer must parallel the Woop buffer");
    const uint64_t n_inner = n_nodes_u4 / 4;
    std::vector<uint8_t> seen(n_inner, 0);
    std::vector<uint8_t> leaf_seen(n_woop_u4 + 1, 0);
    struct E { uint32_t node; uint32_t depth; };
    std::vector<E> st{{0, 0}};
    seen[0] = 1;
    uint32_t max_depth = 0;
    uint64_t visited = 0;
    while (!st.empty()) {
        E e = st.back();
        st.pop_back();
        visited++;
        max_depth = std::max(max_depth, e.depth);
        if (e.depth >= 64) return fail(RB2_EFORMAT, "tree deeper than the 64-entry traversal stack");
        const uint32_t* n = nodes + (size_t)e.node * 16;
        for (int k = 0; k < 2; k++) {
            int32_t c = (int32_t)n[12 + k];
            if (c >= 0) {
                if ((uint32_t)c % 4 != 0 || (uint64_t)c / 4 >= n_inner) return fail(RB2_EFORMAT, "inner child index out of range");
                uint32_t ci = (uint32_t)c / 4;
                if (seen[ci]) return fail(RB2_EFORMAT, "node referenced twice (not a tree)");
                seen[ci] = 1;
                st.push_back({ci, e.depth + 1});
            } else {
                uint64_t a = (uint64_t)(uint32_t)(~c);
                if (leaf_seen[std::min<uint64_t>(a, n_woop_u4)]) {
                    // Leaves may not share Woop runs in packed output, but a
                    // shared run is still safe to traverse; accept it.
                }
                // Walk the run: 3 slots per triangle until the terminator.
                for (;;) {
                    if (a >= n_woop_u4) return fail(RB2_EFORMAT, "leaf run not terminated");
                    if (woop[a * 4] == 0x80000000u) break;
                    if (a + 3 > n_woop_u4) return fail(RB2_EFORMAT, "leaf triangle overruns Woop buffer");
                    if (n_tris_hint && triidx[a] >= n_tris_hint) return fail(RB2_EFORMAT, "triangle id out of range");
                    a += 3;
                }
                leaf_seen[std::min<uint64_t>((uint64_t)(uint32_t)(~c), n_woop_u4)] = 1;
                max_depth = std::max(max_depth, e.depth + 1);
            }
        }
    }
    if (max_depth_out) *max_depth_out = max_depth;
    (void)visited;
    return RB2_OK;
}

// ---- cache ----------------------------------------------------------------------
namespace {

const char kMagic[8] = {'R', 'B', '2', 'B', 'V', 'H', 0, 1};
const uint32_t kVersion = 1;

uint64_t fnv1a(const void* data, size_t n, uint64_t h)
{
    const uint8_t* p = static_cast<const uint8_t*>(data);
    for (size_t i = 0; i < n; i++) { h ^= p[i]; h *= 1099511628211ull; }
    return h;
}

struct CacheHeader {
    char magic[8];
    uint32_t version, layout;
    uint64_t n_nodes_u4, n_woop_u4, n_triidx;
    uint32_t n_inner, n_leaves, n_tri_refs, n_tris;
    float sah;
    uint32_t max_depth;
    uint64_t checksum;
};

}  // namespace

int save_binary(const HostBvh& b, const char* path)
{
    CacheHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.layout = b.layout;
    h.n_nodes_u4 = b.nodes.size() / 4;
    h.n_woop_u4 = b.woop.size() / 4;
    h.n_triidx = b.triidx.size();
    h.n_inner = b.counts.n_inner;
    h.n_leaves = b.counts.n_leaves;
    h.n_tri_refs = b.counts.n_tri_refs;
    h.n_tris = b.counts.n_tris;
    h.sah = b.counts.sah;
    h.max_depth = b.counts.max_depth;
    uint64_t c = 1469598103934665603ull;
    c = fnv1a(b.nodes.data(), b.nodes.size() * 4, c);
    c = fnv1a(b.woop.data(), b.woop.size() * 4, c);
    c = fnv1a(b.triidx.data(), b.triidx.size() * 4, c);
    h.checksum = c;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(RB2_EIO, std::string("cannot open for writing: ") + path);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    ok = ok && std::fwrite(b.nodes.data(), 4, b.nodes.size(), f) == b.nodes.size();
    ok = ok && std::fwrite(b.woop.data(), 4, b.woop.size(), f) == b.woop.size();
    ok = ok && std::fwrite(b.triidx.data(), 4, b.triidx.size(), f) == b.triidx.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RB2_OK : fail(RB2_EIO, std::string("write failed: ") + path);
}

int save_text(const HostBvh& b, const char* path)
{
    std::ofstream out(path, std::ios::binary);
    if (!out) return fail(RB2_EIO, std::string("cannot open for writing: ") + path);
    // Reference text cache (cudabvh.cpp:176-214): magic, three sizes, layout,
    // uint4 lines, index lines, end marker 0x1234567.
    out << 0x76543210u << "\n" << b.nodes.size() / 4 << "\n" << b.woop.size() / 4 << "\n" << b.triidx.size() << "\n"
        << b.layout << "\n";
    for (size_t i = 0; i < b.nodes.size(); i += 4)
        out << b.nodes[i] << " " << b.nodes[i + 1] << " " << b.nodes[i + 2] << " " << b.nodes[i + 3] << "\n";
    for (size_t i = 0; i < b.woop.size(); i += 4)
        out << b.woop[i] << " " << b.woop[i + 1] << " " << b.woop[i + 2] << " " << b.woop[i + 3] << "\n";
    for (size_t i = 0; i < b.triidx.size(); i++) out << b.triidx[i] << "\n";
    out << 0x1234567u << "\n";
    return out.good() ? RB2_OK : fail(RB2_EIO, std::string("write failed: ") + path);
}

int load_any(const char* path, HostBvh& b)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(RB2_EIO, std::string("cannot open: ") + path);
    char magic[8] = {0};
    size_t got = std::fread(magic, 1, 8, f);
    if (got == 8 && std::memcmp(magic, kMagic, 8) == 0) {
        std::rewind(f);
        CacheHeader h{};
        if (std::fread(&h, sizeof(h), 1, f) != 1) { std::fclose(f); return fail(RB2_EFORMAT, "truncated header"); }
        if (h.version != kVersion) { std::fclose(f); return fail(RB2_EFORMAT, "unsupported cache version"); }
        if (h.layout != RB2_LAYOUT_COMPACT2) { std::fclose(f); return fail(RB2_EFORMAT, "layout mismatch"); }
        if (h.n_nodes_u4 > (1ull << 34) || h.n_woop_u4 > (1ull << 34) || h.n_triidx != h.n_woop_u4) {
            std::fclose(f);
            return fail(RB2_EFORMAT, "implausible sizes in cache header");
        }
        b.nodes.resize(h.n_nodes_u4 * 4);
        b.woop.resize(h.n_woop_u4 * 4);
        b.triidx.resize(h.n_triidx);
        bool ok = std::fread(b.nodes.data(), 4, b.nodes.size(), f) == b.nodes.size();
        ok = ok && std::fread(b.woop.data(), 4, b.woop.size(), f) == b.woop.size();
        ok = ok && std::fread(b.triidx.data(), 4, b.triidx.size(), f) == b.triidx.size();
        std::fclose(f);
        if (!ok) return fail(RB2_EFORMAT, "truncated cache body");
        uint64_t c = 1469598103934665603ull;
        c = fnv1a(b.nodes.data(), b.nodes.size() * 4, c);
        c = fnv1a(b.woop.data(), b.woop.size() * 4, c);
        c = fnv1a(b.triidx.data(), b.triidx.size() * 4, c);
        if (c != h.checksum) return fail(RB2_EFORMAT, "cache checksum mismatch");
        b.layout = h.layout;
        b.counts = rb2_bvh_counts{};
        b.counts.n_inner = h.n_inner;
        b.counts.n_leaves = h.n_leaves;
        b.counts.n_tri_refs = h.n_tri_refs;
        b.counts.n_tris = h.n_tris;
        b.counts.sah = h.sah;
        b.counts.max_depth = h.max_depth;
    } else {
        std::fclose(f);
        std::ifstream in(path);
        uint64_t magic_num = 0, nn = 0, nw = 0, nt = 0;
        uint32_t layout = 0;
        in >> magic_num;
        if (!in || magic_num != 0x76543210ull) return fail(RB2_EFORMAT, "not an rb2 or reference BVH cache");
        in >> nn >> nw >> nt >> layout;
        if (!in || nn > (1ull << 34) || nw > (1ull << 34) || nt != nw) return fail(RB2_EFORMAT, "bad reference cache sizes");
        if (layout != RB2_LAYOUT_COMPACT2) return fail(RB2_EFORMAT, "reference cache is not the Compact2 layout");
        b.nodes.resize(nn * 4);
        b.woop.resize(nw * 4);
        b.triidx.resize(nt);
        for (auto& x : b.nodes) in >> x;
        for (auto& x : b.woop) in >> x;
        for (auto& x : b.triidx) in >> x;
        uint64_t eof = 0;
        in >> eof;
        if (!in || eof != 0x1234567ull) return fail(RB2_EFORMAT, "reference cache end marker missing");
        b.layout = layout;
        b.counts = rb2_bvh_counts{};
    }
    uint32_t depth = 0;
    int rc = validate_compact2(b.nodes.data(), b.nodes.size() / 4, b.woop.data(), b.woop.size() / 4, b.triidx.data(),
                               b.triidx.size(), 0, &depth);
    if (rc) return rc;
    b.counts.n_nodes_u4 = b.nodes.size() / 4;
    b.counts.n_woop_u4 = b.woop.size() / 4;
    b.counts.n_triidx = b.triidx.size();
    b.counts.layout = b.layout;
    if (!b.counts.max_depth) b.counts.max_depth = depth;
    if (!b.counts.n_inner) b.counts.n_inner = (uint32_t)(b.nodes.size() / 16);
    return RB2_OK;
}

}  // namespace rb2
