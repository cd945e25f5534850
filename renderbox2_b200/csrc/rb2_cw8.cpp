// Compressed 8-wide node layout (RB2_NODE_ORDER_CW8), collapsed on the host
// from a binary Compact2 tree (the reference's layout,
// accelerators/sbvh/cudabvh.cpp:216-296).
//
// The node format follows the compressed wide BVH of Ylitie, Karras and
// Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide
// BVHs" (HPG 2017): eight child boxes quantized to 8 bits per plane in a
// per-node grid (origin p, power-of-two scale per axis), inner children
// stored contiguously from child_base and leaf triangles contiguously from
// tri_base, child slots assigned by ray octant so
// that visiting hit children in bit order is roughly front to back, and the
// binary tree's subtrees distributed over slots by the paper's SAH dynamic
// program.  Node
// words (80 bytes, 5 x uint4):
//   [0..2]  p.xyz (float)
//   [3]     exponent bytes ex | ey << 8 | ez << 16 (biased by 127), imask << 24
//   [4]     child_base (node index)     [5] tri_base (triangle index)
//   [6]     triangle mask: bits 3s .. 3s + n - 1 set for a leaf slot s of n (1-3)
//           triangles; triangle bit b is triangle tri_base + popc(mask below b)
//           (triangles stored in slot order)    [7] unused
// (In place of the paper's per-slot meta bytes: the traversal then builds its
// node and triangle masks from the 8-bit mask of hit slots with two table
// lookups instead of decoding a byte per child.)
//   [8..9]  qlo.x[8]   [10..11] qhi.x[8]
//   [12..13] qlo.y[8]  [14..15] qhi.y[8]
//   [16..17] qlo.z[8]  [18..19] qhi.z[8]
// Quantized boxes contain the binary boxes plus a margin of 2^-16 x the
// scene's largest coordinate (several times the rounding error of either slab
// test for rays that start inside the scene's coordinate range) plus 2^-14 of
// the parent node's extent (the plane decode's offset rounding), so a box the
// binary traversal enters is entered here too despite the different rounding
// of the two slab tests; closest hits therefore equal the binary traversal's
// except for exact ties in t (and for axis-parallel rays that run exactly in a
// binary box's boundary plane, which the binary slab test culls).
#include <algorithm>
#include <cmath>

#include "rb2_internal.h"

namespace rb2 {
namespace {

constexpr uint32_t kTerm = 0x80000000u;

struct Item {
    int32_t node = -1;            // binary inner node index, or -1: triangle refs
    uint32_t ref0 = 0, nref = 0;  // range in the refs pool (node == -1)
    bool demote = false;          // ref list placed as an inner child (its own wide node)
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

struct Pending {                  // a wide node to emit
    int32_t node;                 // binary node to expand, or -1: split refs
    uint32_t ref0, nref;
    double lo[3], hi[3];          // box of a ref list (node == -1)
    uint32_t level;
};

uint32_t slots_of(const Item& it)
{
    if (it.node >= 0) return 1;
    return (it.nref + 2) / 3;
}

// A box that bounds nothing (inverted or not finite) is never entered.
bool box_valid(const Item& it)
{
    for (int a = 0; a < 3; a++)
        if (!(it.lo[a] <= it.hi[a]) || !std::isfinite(it.lo[a]) || !std::isfinite(it.hi[a])) return false;
    return true;
}

double area_of(const Item& it)
{
    const double dx = it.hi[0] - it.lo[0], dy = it.hi[1] - it.lo[1], dz = it.hi[2] - it.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

struct Collapser {
    const uint32_t* bn;
    const uint32_t* woop;
    const uint32_t* triidx;
    double margin = 0.0;
    std::vector<uint32_t> refs;   // Woop float4 offsets of leaf triangles
    Cw8Layout* out = nullptr;

    uint32_t count_refs(uint32_t w) const
    {
        uint32_t n = 0;
        while (woop[(size_t)w * 4] != kTerm) { n++; w += 3; }
        return n;
    }

    Item child(uint32_t b, int k, bool materialize)
    {
        const uint32_t* w = bn + (size_t)b * 16;
        Item it;
        const int32_t c = (int32_t)w[12 + k];
        const int xo = k ? 4 : 0, zo = k ? 10 : 8;
        it.lo[0] = u2f(w[xo + 0]); it.hi[0] = u2f(w[xo + 1]);
        it.lo[1] = u2f(w[xo + 2]); it.hi[1] = u2f(w[xo + 3]);
        it.lo[2] = u2f(w[zo + 0]); it.hi[2] = u2f(w[zo + 1]);
        if (c >= 0) {
            it.node = c / 4;
        } else {
            uint32_t wo = ~(uint32_t)c;
            it.nref = count_refs(wo);
            if (materialize) {
                it.ref0 = (uint32_t)refs.size();
                for (uint32_t i = 0; i < it.nref; i++, wo += 3) refs.push_back(wo);
            }
        }
        return it;
    }

    // ---- SAH-optimal use of a wide node's eight slots: the dynamic program of
    // Ylitie et al. (section 4.1) over this tree's fixed leaves.  cost(b, j) is
    // the cost of subtree b placed in at most j slots of a parent: one inner
    // slot (a wide node rooted at b: area x kCostNode + its children's best
    // split of eight slots), or its two children sharing the j slots.  A leaf
    // of k refs costs area x kCostTri x k inline (ceil(k / 3) slots), or as a
    // demoted ref list in one slot, area x (kCostNode + kCostTri x k).
    static constexpr double kCostNode = 1.0, kCostTri = 0.3;
    std::vector<float> dcost;     // 9 per inner node (j = 1..8)
    std::vector<uint8_t> dsplit;  // 9 per inner node: 0 one inner slot, i: i slots to child 0
    std::vector<uint8_t> nsplit;  // per inner node: child 0's slots in a wide node rooted there

    double ccost(const Item& it, uint32_t j) const
    {
        if (it.node >= 0) return dcost[(size_t)it.node * 9 + j];
        if (it.nref == 0) return 0.0;
        const double a = area_of(it);
        return slots_of(it) <= j ? a * kCostTri * it.nref : a * (kCostNode + kCostTri * it.nref);
    }

    void plan_costs()
    {
        std::vector<uint32_t> order{0};
        for (size_t h = 0; h < order.size(); h++)
            for (int k = 0; k < 2; k++) {
                const int32_t c = (int32_t)bn[(size_t)order[h] * 16 + 12 + k];
                if (c >= 0) order.push_back((uint32_t)c / 4);
            }
        uint32_t n_inner = 0;
        for (uint32_t b : order) n_inner = std::max(n_inner, b + 1);
        dcost.assign((size_t)n_inner * 9, 0.0f);
        dsplit.assign((size_t)n_inner * 9, 0);
        nsplit.assign(n_inner, 1);
        for (size_t h = order.size(); h-- > 0;) {
            const uint32_t b = order[h];
            const Item c0 = child(b, 0, false), c1 = child(b, 1, false);
            Item u = c0;
            for (int a = 0; a < 3; a++) { u.lo[a] = std::min(c0.lo[a], c1.lo[a]); u.hi[a] = std::max(c0.hi[a], c1.hi[a]); }
            const double area = box_valid(u) ? area_of(u) : 0.0;
            double best = INFINITY;
            for (uint32_t i = 1; i < 8; i++) {
                const double v = ccost(c0, i) + ccost(c1, 8 - i);
                if (v < best) { best = v; nsplit[b] = (uint8_t)i; }
            }
            const double cnode = area * kCostNode + best;
            dcost[(size_t)b * 9 + 1] = (float)cnode;
            for (uint32_t j = 2; j <= 8; j++) {
                double v = cnode;
                uint8_t s = 0;
                for (uint32_t i = 1; i < j; i++) {
                    const double w = ccost(c0, i) + ccost(c1, j - i);
                    if (w < v) { v = w; s = (uint8_t)i; }
                }
                dcost[(size_t)b * 9 + j] = (float)v;
                dsplit[(size_t)b * 9 + j] = s;
            }
        }
    }

    void distribute(Item it, uint32_t j, std::vector<Item>& out)
    {
        if (it.node < 0) {
            it.demote = slots_of(it) > j;
            out.push_back(it);
            return;
        }
        const uint8_t s = dsplit[(size_t)it.node * 9 + j];
        if (s == 0) { out.push_back(it); return; }
        distribute(child((uint32_t)it.node, 0, true), s, out);
        distribute(child((uint32_t)it.node, 1, true), j - s, out);
    }

    // The entries of the wide node rooted at binary node b.
    std::vector<Item> plan(uint32_t b)
    {
        std::vector<Item> items;
        const uint32_t s = nsplit[b];
        distribute(child(b, 0, true), s, items);
        distribute(child(b, 1, true), 8 - s, items);
        items.erase(std::remove_if(items.begin(), items.end(), [](const Item& it) { return it.node < 0 && it.nref == 0; }),
                    items.end());
        return items;
    }

    // A list of triangle refs sharing one box: up to 24 refs fill leaf slots
    // directly; longer lists split into eight ref lists (placed as inner children).
    std::vector<Item> split(const Pending& p)
    {
        std::vector<Item> items;
        const uint32_t parts = p.nref <= 24 ? 1u : 8u;
        const uint32_t per = (p.nref + parts - 1) / parts;
        for (uint32_t r = 0; r < p.nref; r += per) {
            Item it;
            it.ref0 = p.ref0 + r;
            it.nref = std::min(per, p.nref - r);
            std::copy(p.lo, p.lo + 3, it.lo);
            std::copy(p.hi, p.hi + 3, it.hi);
            items.push_back(it);
        }
        return items;
    }

    void emit(std::vector<Item> items, uint32_t level, std::vector<Pending>& queue);
};

float round_down(double x)
{
    float f = (float)x;
    if ((double)f > x) f = std::nextafter(f, -INFINITY);
    return f;
}

void Collapser::emit(std::vector<Item> items, uint32_t level, std::vector<Pending>& queue)
{
    // Demote the largest leaf to an inner child until eight slots suffice.
    std::vector<char> demoted(items.size(), 0);
    for (size_t i = 0; i < items.size(); i++) demoted[i] = items[i].demote ? 1 : 0;
    for (;;) {
        uint32_t slots = 0;
        for (size_t i = 0; i < items.size(); i++) slots += demoted[i] ? 1 : slots_of(items[i]);
        if (slots <= 8) break;
        // Only a leaf of more than 3 refs takes more than one slot, and with at
        // most eight items one such leaf exists whenever slots exceed eight.
        int big = -1;
        for (int i = 0; i < (int)items.size(); i++)
            if (items[i].node < 0 && !demoted[i] && items[i].nref > 3 && (big < 0 || items[i].nref > items[big].nref))
                big = i;
        if (big < 0) break;
        demoted[big] = 1;
    }
    // Slot entries: inner children (binary node or demoted ref list), and leaf chunks of up to 3 refs.
    struct Slot {
        int item;
        bool inner;
        uint32_t ref0, nref;
    };
    std::vector<Slot> entries;
    entries.reserve(8);
    for (int i = 0; i < (int)items.size(); i++) {
        if (items[i].node >= 0 || demoted[i]) { entries.push_back({i, true, 0, 0}); continue; }
        for (uint32_t r = 0; r < items[i].nref; r += 3)
            entries.push_back({i, false, items[i].ref0 + r, std::min<uint32_t>(3, items[i].nref - r)});
    }
    double ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (const Item& it : items)
        if (box_valid(it))
            for (int a = 0; a < 3; a++) { ulo[a] = std::min(ulo[a], it.lo[a]); uhi[a] = std::max(uhi[a], it.hi[a]); }
    if (!(ulo[0] <= uhi[0]))
        for (int a = 0; a < 3; a++) ulo[a] = uhi[a] = 0.0;
    // Octant slot assignment: slot s takes the entry met first by rays whose
    // direction signs are s (bit a set: negative along axis a).
    int slot_of_entry[8], entry_of_slot[8];
    std::fill(slot_of_entry, slot_of_entry + 8, -1);
    std::fill(entry_of_slot, entry_of_slot + 8, -1);
    {
        struct Cost {
            double c;
            int e, s;
        };
        Cost costs[64];  // at most eight entries (the demotion above keeps slots <= 8)
        int nc = 0;
        for (int e = 0; e < (int)entries.size() && e < 8; e++) {
            const Item& it = items[entries[e].item];
            double d[3];
            for (int a = 0; a < 3; a++) d[a] = 0.5 * (it.lo[a] + it.hi[a]) - 0.5 * (ulo[a] + uhi[a]);
            for (int s = 0; s < 8; s++) {
                const double c = (s & 1 ? -d[0] : d[0]) + (s & 2 ? -d[1] : d[1]) + (s & 4 ? -d[2] : d[2]);
                costs[nc++] = {c, e, s};
            }
        }
        // Ties in cost resolve in (entry, slot) order.
        std::sort(costs, costs + nc, [](const Cost& a, const Cost& b) {
            return a.c < b.c || (a.c == b.c && (a.e < b.e || (a.e == b.e && a.s < b.s)));
        });
        for (int k = 0; k < nc; k++) {
            const Cost& c = costs[k];
            if (slot_of_entry[c.e] < 0 && entry_of_slot[c.s] < 0) { slot_of_entry[c.e] = c.s; entry_of_slot[c.s] = c.e; }
        }
    }
    // Quantization grid.  Each child box is widened by the scene margin and by
    // 2^-14 of this node's extent per axis: the traversal decodes a plane as
    // the float 32768 + q and folds 32768 cells into its slab offset, whose
    // rounding is at most about 1/512 of a cell (2^-17 of the node).
    float p[3];
    int ex[3];
    double scale[3], wid[3];
    for (int a = 0; a < 3; a++) {
        wid[a] = std::max(0.0, uhi[a] - ulo[a]) * 0x1p-14;
        p[a] = round_down(ulo[a] - margin - wid[a]);
        const double ext = (uhi[a] + margin + wid[a]) - (double)p[a];
        int e = -126;
        if (ext > 0.0) {
            e = (int)std::ceil(std::log2(ext / 255.0));
            while (std::ldexp(255.0, e) < ext) e++;
            while (e > -126 && std::ldexp(255.0, e - 1) >= ext) e--;
        }
        ex[a] = std::max(-126, std::min(127, e));
        scale[a] = std::ldexp(1.0, ex[a]);
    }
    const size_t base = out->nodes.size();
    out->nodes.resize(base + 20, 0u);
    uint32_t* w = &out->nodes[base];
    w[0] = f2u(p[0]); w[1] = f2u(p[1]); w[2] = f2u(p[2]);
    uint32_t imask = 0;
    const uint32_t child_base = (uint32_t)queue.size();
    const uint32_t tri_base = out->n_tris;
    uint8_t qlo[3][8], qhi[3][8];
    uint32_t tmask = 0;
    for (int a = 0; a < 3; a++)
        for (int s = 0; s < 8; s++) { qlo[a][s] = 255; qhi[a][s] = 0; }
    for (int s = 0; s < 8; s++) {
        const int e = entry_of_slot[s];
        if (e < 0) continue;
        const Slot& sl = entries[e];
        const Item& it = items[sl.item];
        for (int a = 0; a < 3 && box_valid(it); a++) {
            const double lo = std::floor(((it.lo[a] - margin - wid[a]) - (double)p[a]) / scale[a]);
            const double hi = std::ceil(((it.hi[a] + margin + wid[a]) - (double)p[a]) / scale[a]);
            qlo[a][s] = (uint8_t)std::max(0.0, std::min(255.0, lo));
            qhi[a][s] = (uint8_t)std::max(0.0, std::min(255.0, hi));
        }
        if (sl.inner) {
            imask |= 1u << s;
            Pending q{};
            q.node = it.node;
            q.level = level + 1;
            if (it.node < 0) {
                q.ref0 = it.ref0;
                q.nref = it.nref;
                std::copy(it.lo, it.lo + 3, q.lo);
                std::copy(it.hi, it.hi + 3, q.hi);
            }
            queue.push_back(q);
        } else {
            tmask |= ((1u << sl.nref) - 1u) << (3 * s);
            for (uint32_t r = 0; r < sl.nref; r++) {
                const uint32_t wo = refs[sl.ref0 + r];
                out->woop.insert(out->woop.end(), woop + (size_t)wo * 4, woop + (size_t)wo * 4 + 12);
                out->triidx.push_back(triidx[wo]);
            }
            out->n_tris += sl.nref;
        }
    }
    w[3] = (uint32_t)(ex[0] + 127) | ((uint32_t)(ex[1] + 127) << 8) | ((uint32_t)(ex[2] + 127) << 16) | (imask << 24);
    w[4] = child_base;
    w[5] = tri_base;
    w[6] = tmask;
    w[7] = 0;
    for (int a = 0; a < 3; a++)
        for (int s = 0; s < 8; s++) {
            w[8 + 4 * a + s / 4] |= (uint32_t)qlo[a][s] << (8 * (s % 4));
            w[10 + 4 * a + s / 4] |= (uint32_t)qhi[a][s] << (8 * (s % 4));
        }
    out->depth = std::max(out->depth, level + 1);
}

}  // namespace

int collapse_cw8(const uint32_t* nodes, uint64_t n_nodes_u4, const uint32_t* woop, const uint32_t* triidx, Cw8Layout& out)
{
    out = Cw8Layout();
    if (n_nodes_u4 < 4) return fail(RB2_EINVAL, "BVH has no inner node");
    Collapser c;
    c.bn = nodes;
    c.woop = woop;
    c.triidx = triidx;
    c.out = &out;
    // Size hints from the binary inner-node count (about 3 per wide node,
    // about 3 triangle refs per binary leaf).
    const size_t n_inner = (size_t)(n_nodes_u4 / 4);
    out.nodes.reserve((n_inner / 3 + 1) * 20);
    out.woop.reserve((n_inner + 1) * 3 * 12);
    out.triidx.reserve((n_inner + 1) * 3);
    double m = 0.0;
    for (int k = 0; k < 2; k++) {
        const Item r = c.child(0, k, false);
        for (int a = 0; a < 3; a++) m = std::max(m, std::max(std::fabs(r.lo[a]), std::fabs(r.hi[a])));
    }
    c.margin = std::max(m * 0x1p-16, 1e-30);
    c.plan_costs();
    // Breadth-first: a node's inner children are queued together, so they are
    // contiguous from its child_base.
    std::vector<Pending> queue;
    Pending root{};
    root.node = 0;
    queue.push_back(root);
    for (size_t h = 0; h < queue.size(); h++) {
        const Pending pd = queue[h];
        std::vector<Item> items = pd.node >= 0 ? c.plan((uint32_t)pd.node) : c.split(pd);
        c.emit(std::move(items), pd.level, queue);
    }
    out.n_nodes = (uint32_t)(out.nodes.size() / 20);
    return RB2_OK;
}

}  // namespace rb2

namespace rb2 {
const HostBvh& host_of(const rb2_host_bvh* b);
}  // namespace rb2

extern "C" int rb2_bvh_cw8_layout(const rb2_host_bvh* bvh, rb2_cw8_counts* counts, uint32_t* nodes, uint32_t* woop,
                                  uint32_t* triidx)
{
    using namespace rb2;
    if (!bvh || !counts) return fail(RB2_EINVAL, "null argument");
    try {
        const HostBvh& h = host_of(bvh);
        int rc = validate_compact2(h.nodes.data(), h.nodes.size() / 4, h.woop.data(), h.woop.size() / 4, h.triidx.data(),
                                   h.triidx.size(), 0, nullptr);
        if (rc) return rc;
        Cw8Layout cw;
        rc = collapse_cw8(h.nodes.data(), h.nodes.size() / 4, h.woop.data(), h.triidx.data(), cw);
        if (rc) return rc;
        counts->n_nodes = cw.n_nodes;
        counts->n_tris = cw.n_tris;
        counts->depth = cw.depth;
        counts->reserved = 0;
        if (nodes) std::copy(cw.nodes.begin(), cw.nodes.end(), nodes);
        if (woop) std::copy(cw.woop.begin(), cw.woop.end(), woop);
        if (triidx) std::copy(cw.triidx.begin(), cw.triidx.end(), triidx);
        return RB2_OK;
    } catch (const std::bad_alloc&) {
        return fail(RB2_ENOMEM, "host allocation failed in the 8-wide collapse");
    }
}
