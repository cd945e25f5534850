// Host SBVH builder (spatial-split BVH, Stich, Friedrich & Dietrich, "Spatial
// Splits in Bounding Volume Hierarchies", HPG 2009).
//
// Same split semantics as the reference's SplitBVHBuilder
// (accelerators/sbvh/splitbvhbuilder.cpp:234-626): SAH with node cost 2*A and
// triangle cost n*A, degenerate-reference removal, spatial splits only where
// the best object split's child overlap is at least alpha * root area and the
// depth is below the spatial limit, chopped spatial binning with
// unsplit/duplicate decisions per straddling reference, leaves when the leaf
// SAH wins.  Different engineering, chosen for a many-core host:
//   - object splits are binned (Wald 2007) above `exact_sweep_max` references
//     and exact sorted sweeps below it;
//   - binning of large nodes is split across threads, subtrees are built
//     fork-join on a bounded thread budget (std::thread, no OpenMP runtime);
//   - each node owns its reference array (no shared reference stack), so
//     subtrees never touch each other's memory.
#include "rb2_internal.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <thread>

namespace rb2 {
namespace {

struct Ref {
    uint32_t tri;
    Box box;
};

struct BNode {
    Box box;
    std::unique_ptr<BNode> c[2];
    std::vector<uint32_t> tris;
    bool leaf = false;
};

struct ObjectSplit {
    float sah = FLT_MAX;
    int dim = 0;
    uint32_t num_left = 0;
    bool binned = false;
    float bin_origin = 0.0f, bin_scale = 0.0f;  // binned: bin(c) = (c - origin) * scale
    int bin_count = 0;
    int bin_split = 0;                          // binned: left = bins [0, bin_split)
    Box left, right;
};

struct SpatialSplit {
    float sah = FLT_MAX;
    int dim = 0;
    float pos = 0.0f;
};

struct SpatialBin {
    Box box;
    uint32_t enter = 0, exit = 0;
};

class Builder {
public:
    Builder(const float* v, const uint32_t* idx, const rb2_build_params& p)
        : V_(reinterpret_cast<const f3*>(v)), I_(idx), p_(p)
    {
        unsigned hw = std::thread::hardware_concurrency();
        max_threads_ = p.num_threads > 0 ? (unsigned)p.num_threads : (hw ? hw : 1);
    }

    std::unique_ptr<BNode> run(uint32_t ntri)
    {
        std::vector<Ref> refs(ntri);
        Box root;
        parallel_chunks(ntri, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; i++) {
                Ref& r = refs[i];
                r.tri = (uint32_t)i;
                r.box = Box();
                r.box.insert(vtx(i, 0));
                r.box.insert(vtx(i, 1));
                r.box.insert(vtx(i, 2));
            }
        });
        for (const Ref& r : refs) root.grow(r.box);
        min_overlap_ = root.area() * p_.split_alpha;
        return build(std::move(refs), root, 0);
    }

    uint32_t duplicates() const { return dups_.load(); }

private:
    const f3* V_;
    const uint32_t* I_;
    rb2_build_params p_;
    float min_overlap_ = 0.0f;
    unsigned max_threads_ = 1;
    std::atomic<unsigned> busy_{1};
    std::atomic<uint32_t> dups_{0};

    f3 vtx(size_t tri, int k) const { return V_[I_[3 * tri + k]]; }
    float tri_cost(uint32_t n) const { return (float)n * p_.sah_triangle_cost; }
    float node_cost(uint32_t n) const { return (float)n * p_.sah_node_cost; }

    // Runs fn(begin, end) over [0, n) on up to max_threads_ threads when n is large.
    template <class F>
    void parallel_chunks(size_t n, F&& fn, size_t min_chunk = 65536)
    {
        unsigned nt = (unsigned)std::min<size_t>(max_threads_, (n + min_chunk - 1) / min_chunk);
        if (nt <= 1) { fn(0, n); return; }
        std::vector<std::thread> th;
        size_t step = (n + nt - 1) / nt;
        for (unsigned t = 1; t < nt; t++) {
            size_t b = t * step, e = std::min(n, b + step);
            if (b < e) th.emplace_back([&fn, b, e] { fn(b, e); });
        }
        fn(0, std::min(n, step));
        for (auto& x : th) x.join();
    }

    std::unique_ptr<BNode> make_leaf(const std::vector<Ref>& refs, const Box& box)
    {
        auto n = std::make_unique<BNode>();
        n->leaf = true;
        n->box = box;
        // The reference pops references off the end of its stack (create_leaf,
        // splitbvhbuilder.cpp:359-367), so a leaf lists them in reverse order.
        n->tris.reserve(refs.size());
        for (size_t i = refs.size(); i-- > 0;) n->tris.push_back(refs[i].tri);
        return n;
    }

    static bool degenerate(const Box& b)
    {
        f3 s = b.hi - b.lo;
        float mn = std::min(s.x, std::min(s.y, s.z));
        float mx = std::max(s.x, std::max(s.y, s.z));
        return mn < 0.0f || (s.x + s.y + s.z) == mx;
    }

    std::unique_ptr<BNode> build(std::vector<Ref>&& refs, Box bounds, int depth)
    {
        // Remove degenerates (splitbvhbuilder.cpp:300-316).
        refs.erase(std::remove_if(refs.begin(), refs.end(), [](const Ref& r) { return degenerate(r.box); }),
                   refs.end());
        const uint32_t n = (uint32_t)refs.size();
        if (n <= p_.min_leaf_size || depth >= (int)p_.max_depth) return make_leaf(refs, bounds);

        const float area = bounds.area();
        const float leaf_sah = area * tri_cost(n);
        const float node_sah = area * node_cost(2);
        ObjectSplit object = find_object_split(refs, node_sah);

        SpatialSplit spatial;
        if (depth < (int)p_.max_spatial_depth && p_.spatial_bins >= 2) {
            Box overlap = object.left;
            overlap.clip(object.right);
            if (overlap.area() >= min_overlap_) spatial = find_spatial_split(refs, bounds, node_sah);
        }

        const float min_sah = std::min(leaf_sah, std::min(object.sah, spatial.sah));
        if (min_sah == leaf_sah && n <= p_.max_leaf_size) return make_leaf(refs, bounds);

        std::vector<Ref> left, right;
        Box lbox, rbox;
        if (min_sah == spatial.sah) perform_spatial_split(refs, spatial, left, right, lbox, rbox);
        if (left.empty() || right.empty()) {
            left.clear();
            right.clear();
            perform_object_split(refs, object, left, right);
            lbox = object.left;
            rbox = object.right;
        }
        if (left.size() + right.size() > n) dups_ += (uint32_t)(left.size() + right.size() - n);
        std::vector<Ref>().swap(refs);

        auto node = std::make_unique<BNode>();
        node->box = bounds;
        const size_t big = 8192;
        if (left.size() + right.size() > 2 * big && busy_.load() < max_threads_) {
            busy_++;
            std::unique_ptr<BNode> rchild;
            std::thread th([&] { rchild = build(std::move(right), rbox, depth + 1); });
            node->c[0] = build(std::move(left), lbox, depth + 1);
            th.join();
            busy_--;
            node->c[1] = std::move(rchild);
        } else {
            node->c[0] = build(std::move(left), lbox, depth + 1);
            node->c[1] = build(std::move(right), rbox, depth + 1);
        }
        return node;
    }

    // ---- object split -----------------------------------------------------------
    ObjectSplit find_object_split(std::vector<Ref>& refs, float node_sah)
    {
        if (refs.size() <= p_.exact_sweep_max) return exact_object_split(refs, node_sah);
        return binned_object_split(refs, node_sah);
    }

    static float centroid2(const Ref& r, int d) { return get(r.box.lo, d) + get(r.box.hi, d); }

    ObjectSplit exact_object_split(std::vector<Ref>& refs, float node_sah)
    {
        ObjectSplit best;
        const uint32_t n = (uint32_t)refs.size();
        float best_tie = FLT_MAX;
        std::vector<Box> rb(n);
        for (int d = 0; d < 3; d++) {
            std::sort(refs.begin(), refs.end(), [d](const Ref& a, const Ref& b) {
                float ca = centroid2(a, d), cb = centroid2(b, d);
                return ca < cb || (ca == cb && a.tri < b.tri);
            });
            Box acc;
            for (uint32_t i = n - 1; i > 0; i--) { acc.grow(refs[i].box); rb[i - 1] = acc; }
            Box lb;
            for (uint32_t i = 1; i < n; i++) {
                lb.grow(refs[i - 1].box);
                float sah = node_sah + lb.area() * tri_cost(i) + rb[i - 1].area() * tri_cost(n - i);
                float tie = (float)i * (float)i + (float)(n - i) * (float)(n - i);
                if (sah < best.sah || (sah == best.sah && tie < best_tie)) {
                    best.sah = sah;
                    best.dim = d;
                    best.num_left = i;
                    best.left = lb;
                    best.right = rb[i - 1];
                    best_tie = tie;
                }
            }
        }
        return best;
    }

    ObjectSplit binned_object_split(std::vector<Ref>& refs, float node_sah)
    {
        const int B = (int)std::max<uint32_t>(4, std::min<uint32_t>(p_.object_bins, 1024));
        const size_t n = refs.size();
        // Centroid bounds (doubled centroids, like the sort key).
        Box cb;
        for (const Ref& r : refs) cb.insert(mk(centroid2(r, 0), centroid2(r, 1), centroid2(r, 2)));
        struct Bin { Box box; uint32_t cnt = 0; };
        const unsigned nt = (unsigned)std::min<size_t>(max_threads_, std::max<size_t>(1, n / 65536));
        std::vector<Bin> bins((size_t)nt * 3 * B);
        float origin[3], scale[3];
        for (int d = 0; d < 3; d++) {
            float ext = get(cb.hi, d) - get(cb.lo, d);
            origin[d] = get(cb.lo, d);
            scale[d] = ext > 0.0f ? (float)B * 0.99999f / ext : 0.0f;
        }
        auto bin_of = [&](const Ref& r, int d) {
            int b = (int)((centroid2(r, d) - origin[d]) * scale[d]);
            return std::min(B - 1, std::max(0, b));
        };
        {
            std::vector<std::thread> th;
            size_t step = (n + nt - 1) / nt;
            auto work = [&](unsigned t) {
                Bin* my = &bins[(size_t)t * 3 * B];
                size_t b = t * step, e = std::min(n, b + step);
                for (size_t i = b; i < e; i++)
                    for (int d = 0; d < 3; d++) {
                        Bin& x = my[d * B + bin_of(refs[i], d)];
                        x.box.grow(refs[i].box);
                        x.cnt++;
                    }
            };
            for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
            work(0);
            for (auto& x : th) x.join();
            for (unsigned t = 1; t < nt; t++)
                for (int k = 0; k < 3 * B; k++) {
                    bins[k].box.grow(bins[(size_t)t * 3 * B + k].box);
                    bins[k].cnt += bins[(size_t)t * 3 * B + k].cnt;
                }
        }
        ObjectSplit best;
        best.binned = true;
        best.bin_count = B;
        float best_tie = FLT_MAX;
        std::vector<Box> rb(B);
        std::vector<uint32_t> rc(B);
        for (int d = 0; d < 3; d++) {
            if (scale[d] == 0.0f) continue;
            Bin* bd = &bins[d * B];
            Box acc;
            uint32_t cnt = 0;
            for (int i = B - 1; i > 0; i--) { acc.grow(bd[i].box); cnt += bd[i].cnt; rb[i - 1] = acc; rc[i - 1] = cnt; }
            Box lb;
            uint32_t lc = 0;
            for (int i = 1; i < B; i++) {
                lb.grow(bd[i - 1].box);
                lc += bd[i - 1].cnt;
                if (lc == 0 || rc[i - 1] == 0) continue;
                float sah = node_sah + lb.area() * tri_cost(lc) + rb[i - 1].area() * tri_cost(rc[i - 1]);
                float tie = (float)lc * (float)lc + (float)rc[i - 1] * (float)rc[i - 1];
                if (sah < best.sah || (sah == best.sah && tie < best_tie)) {
                    best.sah = sah;
                    best.dim = d;
                    best.num_left = lc;
                    best.bin_split = i;
                    best.bin_origin = origin[d];
                    best.bin_scale = scale[d];
                    best.left = lb;
                    best.right = rb[i - 1];
                    best_tie = tie;
                }
            }
        }
        if (best.sah == FLT_MAX) {
            // All centroids coincide: fall back to a median split by triangle id order.
            ObjectSplit s = exact_median(refs, node_sah);
            return s;
        }
        return best;
    }

    ObjectSplit exact_median(std::vector<Ref>& refs, float node_sah)
    {
        ObjectSplit s;
        const uint32_t n = (uint32_t)refs.size();
        std::sort(refs.begin(), refs.end(), [](const Ref& a, const Ref& b) { return a.tri < b.tri; });
        s.dim = -1;
        s.num_left = n / 2;
        for (uint32_t i = 0; i < n; i++) (i < s.num_left ? s.left : s.right).grow(refs[i].box);
        s.sah = node_sah + s.left.area() * tri_cost(s.num_left) + s.right.area() * tri_cost(n - s.num_left);
        return s;
    }

    void perform_object_split(std::vector<Ref>& refs, const ObjectSplit& s, std::vector<Ref>& left,
                              std::vector<Ref>& right)
    {
        if (s.dim < 0) {  // median by id, refs already in that order
            left.assign(refs.begin(), refs.begin() + s.num_left);
            right.assign(refs.begin() + s.num_left, refs.end());
            return;
        }
        if (!s.binned) {
            const int d = s.dim;
            std::sort(refs.begin(), refs.end(), [d](const Ref& a, const Ref& b) {
                float ca = centroid2(a, d), cb = centroid2(b, d);
                return ca < cb || (ca == cb && a.tri < b.tri);
            });
            left.assign(refs.begin(), refs.begin() + s.num_left);
            right.assign(refs.begin() + s.num_left, refs.end());
            return;
        }
        left.reserve(s.num_left);
        right.reserve(refs.size() - s.num_left);
        for (const Ref& r : refs) {
            int b = (int)((centroid2(r, s.dim) - s.bin_origin) * s.bin_scale);
            b = std::min(s.bin_count - 1, std::max(0, b));
            (b < s.bin_split ? left : right).push_back(r);
        }
    }

    // ---- spatial split ------------------------------------------------------------
    // Clips the triangle of `ref` against the plane x_dim = pos and returns the
    // parts' bounds intersected with the reference's own box
    // (splitbvhbuilder.cpp:586-626).
    void split_reference(const Ref& ref, int dim, float pos, Ref& l, Ref& r) const
    {
        l.tri = r.tri = ref.tri;
        l.box = r.box = Box();
        f3 v1 = vtx(ref.tri, 2);
        for (int i = 0; i < 3; i++) {
            f3 v0 = v1;
            v1 = vtx(ref.tri, i);
            float p0 = get(v0, dim), p1 = get(v1, dim);
            if (p0 <= pos) l.box.insert(v0);
            if (p0 >= pos) r.box.insert(v0);
            if ((p0 < pos && p1 > pos) || (p0 > pos && p1 < pos)) {
                float t = (pos - p0) / (p1 - p0);
                t = fmaxf(0.0f, fminf(t, 1.0f));
                f3 x = v0 + t * (v1 - v0);
                l.box.insert(x);
                r.box.insert(x);
            }
        }
        get(l.box.hi, dim) = pos;
        get(r.box.lo, dim) = pos;
        l.box.clip(ref.box);
        r.box.clip(ref.box);
    }

    SpatialSplit find_spatial_split(const std::vector<Ref>& refs, const Box& bounds, float node_sah)
    {
        const int B = (int)std::min<uint32_t>(p_.spatial_bins, 256);
        const size_t n = refs.size();
        f3 origin = bounds.lo;
        f3 bin_size = (bounds.hi - origin) * (1.0f / (float)B);
        f3 inv = mk(1.0f / bin_size.x, 1.0f / bin_size.y, 1.0f / bin_size.z);
        const unsigned nt = (unsigned)std::min<size_t>(max_threads_, std::max<size_t>(1, n / 32768));
        std::vector<SpatialBin> bins((size_t)nt * 3 * B);
        auto work = [&](unsigned t, size_t b, size_t e) {
            SpatialBin* my = &bins[(size_t)t * 3 * B];
            for (size_t k = b; k < e; k++) {
                const Ref& ref = refs[k];
                for (int d = 0; d < 3; d++) {
                    float bs = get(bin_size, d);
                    if (!(bs > 0.0f)) continue;
                    float o = get(origin, d), iv = get(inv, d);
                    int first = (int)((get(ref.box.lo, d) - o) * iv);
                    int last = (int)((get(ref.box.hi, d) - o) * iv);
                    first = std::min(B - 1, std::max(0, first));
                    last = std::min(B - 1, std::max(first, last));
                    SpatialBin* bd = my + d * B;
                    Ref cur = ref;
                    for (int i = first; i < last; i++) {
                        Ref l, r;
                        split_reference(cur, d, o + bs * (float)(i + 1), l, r);
                        bd[i].box.grow(l.box);
                        cur = r;
                    }
                    bd[last].box.grow(cur.box);
                    bd[first].enter++;
                    bd[last].exit++;
                }
            }
        };
        {
            std::vector<std::thread> th;
            size_t step = (n + nt - 1) / nt;
            for (unsigned t = 1; t < nt; t++) {
                size_t b = t * step, e = std::min(n, b + step);
                th.emplace_back(work, t, b, e);
            }
            work(0, 0, std::min(n, step));
            for (auto& x : th) x.join();
            for (unsigned t = 1; t < nt; t++)
                for (int k = 0; k < 3 * B; k++) {
                    const SpatialBin& s = bins[(size_t)t * 3 * B + k];
                    bins[k].box.grow(s.box);
                    bins[k].enter += s.enter;
                    bins[k].exit += s.exit;
                }
        }
        SpatialSplit best;
        std::vector<Box> rb(B);
        for (int d = 0; d < 3; d++) {
            if (!(get(bin_size, d) > 0.0f)) continue;
            const SpatialBin* bd = &bins[d * B];
            Box acc;
            for (int i = B - 1; i > 0; i--) { acc.grow(bd[i].box); rb[i - 1] = acc; }
            Box lb;
            uint32_t ln = 0, rn = (uint32_t)n;
            for (int i = 1; i < B; i++) {
                lb.grow(bd[i - 1].box);
                ln += bd[i - 1].enter;
                rn -= bd[i - 1].exit;
                float sah = node_sah + lb.area() * tri_cost(ln) + rb[i - 1].area() * tri_cost(rn);
                if (sah < best.sah) {
                    best.sah = sah;
                    best.dim = d;
                    best.pos = get(origin, d) + get(bin_size, d) * (float)i;
                }
            }
        }
        return best;
    }

    // Reference unsplitting (Stich et al. 2009, section 4.3;
    // splitbvhbuilder.cpp:499-584): straddling references go left, right or
    // are duplicated, whichever gives the lowest SAH given the sides so far.
    void perform_spatial_split(const std::vector<Ref>& refs, const SpatialSplit& s, std::vector<Ref>& left,
                               std::vector<Ref>& right, Box& lbox, Box& rbox)
    {
        const int d = s.dim;
        const float pos = s.pos;
        std::vector<const Ref*> straddle;
        lbox = Box();
        rbox = Box();
        for (const Ref& r : refs) {
            if (get(r.box.hi, d) <= pos) { left.push_back(r); lbox.grow(r.box); }
            else if (get(r.box.lo, d) >= pos) { right.push_back(r); rbox.grow(r.box); }
            else straddle.push_back(&r);
        }
        for (const Ref* rp : straddle) {
            Ref lr, rr;
            split_reference(*rp, d, pos, lr, rr);
            Box lub = lbox, rub = rbox, ldb = lbox, rdb = rbox;
            lub.grow(rp->box);
            rub.grow(rp->box);
            ldb.grow(lr.box);
            rdb.grow(rr.box);
            const uint32_t nl = (uint32_t)left.size(), nr = (uint32_t)right.size();
            float lac = tri_cost(nl), rac = tri_cost(nr), lbc = tri_cost(nl + 1), rbc = tri_cost(nr + 1);
            float unsplit_left = lub.area() * lbc + rbox.area() * rac;
            float unsplit_right = lbox.area() * lac + rub.area() * rbc;
            float duplicate = ldb.area() * lbc + rdb.area() * rbc;
            float mn = std::min(unsplit_left, std::min(unsplit_right, duplicate));
            if (mn == unsplit_left) { lbox = lub; left.push_back(*rp); }
            else if (mn == unsplit_right) { rbox = rub; right.push_back(*rp); }
            else { lbox = ldb; rbox = rdb; left.push_back(lr); right.push_back(rr); }
        }
    }
};

void flatten(BNode* n, Tree& t, int32_t slot, uint32_t depth, uint32_t& max_depth, rb2_bvh_counts& c, double prob,
             double& sah, const rb2_build_params& p)
{
    TreeNode& tn = t.nodes[slot];
    tn.box = n->box;
    max_depth = std::max(max_depth, depth);
    if (n->leaf) {
        tn.tri_begin = (uint32_t)t.tri_refs.size();
        tn.tri_count = (uint32_t)n->tris.size();
        t.tri_refs.insert(t.tri_refs.end(), n->tris.begin(), n->tris.end());
        c.n_leaves++;
        c.n_tri_refs += tn.tri_count;
        sah += prob * (double)((float)tn.tri_count * p.sah_triangle_cost);
        return;
    }
    c.n_inner++;
    sah += prob * (double)(2.0f * p.sah_node_cost);
    float pa = n->box.area();
    for (int k = 0; k < 2; k++) {
        int32_t cs = (int32_t)t.nodes.size();
        t.nodes.emplace_back();
        t.nodes[slot].child[k] = cs;
        double cp = pa > 0.0f ? prob * (double)(n->c[k]->box.area() / pa) : 0.0;
        flatten(n->c[k].get(), t, cs, depth + 1, max_depth, c, cp, sah, p);
    }
}

}  // namespace

int build_tree(const float* v, uint32_t nv, const uint32_t* idx, uint32_t ntri, const rb2_build_params& p,
               Tree& tree, rb2_bvh_counts& counts)
{
    for (uint64_t i = 0; i < 3ull * ntri; i++)
        if (idx[i] >= nv) return fail(RB2_EINVAL, "triangle index out of range");
    Builder b(v, idx, p);
    std::unique_ptr<BNode> root = b.run(ntri);
    // The packed layout needs an inner root (cudabvh.cpp:237); wrap a leaf root
    // with an empty second child that no ray can enter.
    if (root->leaf) {
        auto r = std::make_unique<BNode>();
        r->box = root->box;
        r->c[0] = std::move(root);
        r->c[1] = std::make_unique<BNode>();
        r->c[1]->leaf = true;
        root = std::move(r);
    }
    tree.nodes.clear();
    tree.tri_refs.clear();
    tree.nodes.emplace_back();
    uint32_t max_depth = 0;
    double sah = 0.0;
    counts.n_inner = counts.n_leaves = counts.n_tri_refs = 0;
    flatten(root.get(), tree, 0, 0, max_depth, counts, 1.0, sah, p);
    counts.max_depth = max_depth;
    counts.sah = (float)sah;
    counts.n_tris = ntri;
    return RB2_OK;
}

}  // namespace rb2
