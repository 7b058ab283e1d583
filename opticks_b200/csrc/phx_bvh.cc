// phx_bvh.cc : host builder of the 4-wide BVH that replaces the OptiX IAS/GAS.
//
// The reference hands one AABB per CSGPrim to OptiX (CSGOptiX/GAS_Builder.cc:112-130) and
// one instance per qat4 transform (CSGOptiX/SBT.cc:393-460); OptiX builds the hierarchy.
// Here every (instance, prim) pair becomes one leaf with a world-space box (the corner box of the
// prim's box under the instance transform, overlapped with a box built from the prim's CSG tree
// when the engine supplies one: a tilted PMT's cap and neck bound it far more tightly than its
// whole box does), a binned-SAH binary BVH is built over the leaves and collapsed to 4-wide nodes
// whose child boxes are stored per axis (phx_bvh4_node) so the traversal tests four boxes with
// coalesced loads.
// Boxes are padded so that FP32 slab tests never cull a leaf that the CSG intersector hits.
#include "phx_bvh.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

// SAH build parameters: centroid bins per axis (for nodes above PHX_BVH_EXACT_MAX leaves), largest
// leaf range a node may keep, and the cost of visiting a node relative to one leaf test (0: split
// whenever the SAH sum does not grow).  On
// the 17,612-PMT detector the tree splits down to single leaves for any of these settings.
#ifndef PHX_BVH_BINS
#define PHX_BVH_BINS 64
#endif
// nodes of at most this many leaves take the exact SAH sweep (all split positions) instead of bins;
// the sweep sorts each axis, so it is kept for the lower levels of very large scenes
#ifndef PHX_BVH_EXACT_MAX
#define PHX_BVH_EXACT_MAX 65536
#endif
#ifndef PHX_BVH_MAX_LEAF
#define PHX_BVH_MAX_LEAF 4
#endif
#ifndef PHX_BVH_TRAV_COST
#define PHX_BVH_TRAV_COST 0.0
#endif

namespace {

struct Box {
    double lo[3], hi[3];
    Box() { for (int k = 0; k < 3; k++) { lo[k] = std::numeric_limits<double>::infinity(); hi[k] = -std::numeric_limits<double>::infinity(); } }
    void grow(const Box& b) { for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); } }
    void grow(const double* p) { for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); } }
    bool empty() const { return !(lo[0] <= hi[0]); }
    double area() const
    {
        if (empty()) return 0.0;
        double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node2 {
    Box box;
    int left = -1, right = -1;  // inner: children ; leaf: left=-1
    int first = 0, count = 0;   // leaf range in the reordered leaf list
};

struct Builder {
    std::vector<Box> boxes;
    std::vector<double> cent;   // 3 per leaf
    std::vector<int> idx;
    std::vector<Node2> nodes;
    int max_leaf = PHX_BVH_MAX_LEAF;

    // Exact SAH: every split between consecutive centroids along each axis (prefix and suffix box
    // areas over the sorted leaves); a node of one leaf, or of at most max_leaf leaves whose split
    // does not lower the cost, stays a leaf range.
    int split_exact(int me, int first, int count, int depth)
    {
        double best_cost = std::numeric_limits<double>::infinity();
        int best_axis = -1, best_pos = -1;
        std::vector<int> ord(idx.begin() + first, idx.begin() + first + count);
        std::vector<double> right_area((size_t)count + 1, 0.0);
        for (int ax = 0; ax < 3; ax++) {
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cent[3 * a + ax] < cent[3 * b + ax]; });
            Box r;
            for (int k = count - 1; k >= 1; k--) { r.grow(boxes[ord[k]]); right_area[k] = r.area(); }
            Box l;
            for (int k = 1; k < count; k++) {      // left = ord[0, k), right = ord[k, count)
                l.grow(boxes[ord[k - 1]]);
                const double cost = l.area() * k + right_area[k] * (count - k);
                if (cost < best_cost) { best_cost = cost; best_axis = ax; best_pos = k; }
            }
        }
        const double leaf_cost = nodes[me].box.area() * count;
        best_cost += PHX_BVH_TRAV_COST * nodes[me].box.area();
        if (best_axis < 0 || (count <= max_leaf && best_cost >= leaf_cost)) {
            if (count <= max_leaf || best_axis < 0) {
                if (count > max_leaf) {
                    const int half = count / 2;
                    const int l = build(first, half, depth + 1);
                    const int r = build(first + half, count - half, depth + 1);
                    nodes[me].left = l; nodes[me].right = r;
                    return me;
                }
                nodes[me].first = first; nodes[me].count = count;
                return me;
            }
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cent[3 * a + best_axis] < cent[3 * b + best_axis]; });
        std::copy(ord.begin(), ord.end(), idx.begin() + first);
        const int l = build(first, best_pos, depth + 1);
        const int r = build(first + best_pos, count - best_pos, depth + 1);
        nodes[me].left = l; nodes[me].right = r;
        return me;
    }

    int build(int first, int count, int depth)
    {
        Node2 n;
        for (int i = first; i < first + count; i++) n.box.grow(boxes[idx[i]]);
        int me = (int)nodes.size();
        nodes.push_back(n);
        if (count <= 1 || depth > 60) { nodes[me].first = first; nodes[me].count = count; return me; }
        // centroid bounds
        Box cb;
        for (int i = first; i < first + count; i++) cb.grow(&cent[3 * idx[i]]);
        const int NB = PHX_BVH_BINS;
        double best_cost = std::numeric_limits<double>::infinity();
        int best_axis = -1, best_split = -1;
        if (NB <= 0 || count <= PHX_BVH_EXACT_MAX) return split_exact(me, first, count, depth);
        for (int ax = 0; ax < 3; ax++) {
            double lo = cb.lo[ax], hi = cb.hi[ax];
            if (!(hi > lo)) continue;
            Box bb[PHX_BVH_BINS > 0 ? PHX_BVH_BINS : 1]; int bc[PHX_BVH_BINS > 0 ? PHX_BVH_BINS : 1] = {0};
            double scale = NB / (hi - lo);
            for (int i = first; i < first + count; i++) {
                int b = (int)((cent[3 * idx[i] + ax] - lo) * scale);
                b = std::min(NB - 1, std::max(0, b));
                bc[b]++; bb[b].grow(boxes[idx[i]]);
            }
            Box lb[PHX_BVH_BINS > 0 ? PHX_BVH_BINS : 1]; int lc[PHX_BVH_BINS > 0 ? PHX_BVH_BINS : 1];
            Box acc; int ac = 0;
            for (int b = 0; b < NB; b++) { acc.grow(bb[b]); ac += bc[b]; lb[b] = acc; lc[b] = ac; }
            Box racc; int rc = 0;
            for (int b = NB - 1; b > 0; b--) {
                racc.grow(bb[b]); rc += bc[b];
                int lcount = lc[b - 1];
                if (lcount == 0 || rc == 0) continue;
                double cost = lb[b - 1].area() * lcount + racc.area() * rc;
                if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = b; }
            }
        }
        double leaf_cost = nodes[me].box.area() * count;
        best_cost += PHX_BVH_TRAV_COST * nodes[me].box.area();
        if (best_axis < 0 || (count <= max_leaf && best_cost >= leaf_cost)) {
            if (count <= max_leaf || best_axis < 0) {
                if (count > max_leaf) {
                    // all centroids coincide: split the range in the middle
                    int half = count / 2;
                    int l = build(first, half, depth + 1);
                    int r = build(first + half, count - half, depth + 1);
                    nodes[me].left = l; nodes[me].right = r;
                    return me;
                }
                nodes[me].first = first; nodes[me].count = count;
                return me;
            }
        }
        double lo = cb.lo[best_axis], hi = cb.hi[best_axis];
        double scale = NB / (hi - lo);
        int* mid = std::partition(idx.data() + first, idx.data() + first + count, [&](int i) {
            int b = (int)((cent[3 * i + best_axis] - lo) * scale);
            b = std::min(NB - 1, std::max(0, b));
            return b < best_split;
        });
        int lcount = (int)(mid - (idx.data() + first));
        if (lcount == 0 || lcount == count) lcount = count / 2;
        int l = build(first, lcount, depth + 1);
        int r = build(first + lcount, count - lcount, depth + 1);
        nodes[me].left = l; nodes[me].right = r;
        return me;
    }
};

inline bool is_leaf(const Node2& n) { return n.left < 0; }

void set_child(phx_bvh4_node& out, int c, const Box& b, int child)
{
    out.lo_x[c] = (float)b.lo[0]; out.hi_x[c] = (float)b.hi[0];
    out.lo_y[c] = (float)b.lo[1]; out.hi_y[c] = (float)b.hi[1];
    out.lo_z[c] = (float)b.lo[2]; out.hi_z[c] = (float)b.hi[2];
    out.child[c] = child;
}

void set_empty(phx_bvh4_node& out, int c)
{
    out.lo_x[c] = out.lo_y[c] = out.lo_z[c] = 1e30f;
    out.hi_x[c] = out.hi_y[c] = out.hi_z[c] = -1e30f;
    out.child[c] = 0;
}

}  // namespace

// corners of the prim box mapped to world by a row-vector 4x4 (rows q0..q3), in double
static Box world_box(const float* bb6, const float* m)
{
    Box b;
    for (int i = 0; i < 8; i++) {
        double p[3] = { (i & 1) ? bb6[3] : bb6[0], (i & 2) ? bb6[4] : bb6[1], (i & 4) ? bb6[5] : bb6[2] };
        double w[3];
        for (int k = 0; k < 3; k++) w[k] = m[0 * 4 + k] * p[0] + m[1 * 4 + k] * p[1] + m[2 * 4 + k] * p[2] + m[3 * 4 + k];
        b.grow(w);
    }
    return b;
}

int phx_build_bvh4(const std::vector<PhxLeafInput>& in, PhxBvh4Result& out, double global_frac, int max_global)
{
    const int n_all = (int)in.size();
    out.nodes.clear();
    out.leaves.clear();
    out.globals.clear();
    out.leaf_sphere.clear();
    out.global_sphere.clear();
    out.cull[0] = out.cull[1] = out.cull[2] = out.cull[3] = 0.f;
    std::vector<Box> all(n_all);
    Box scene;
    for (int i = 0; i < n_all; i++) {
        Box b = world_box(in[i].bbox, in[i].xform);
        if (in[i].has_wbox) {
            Box t = b;
            for (int k = 0; k < 3; k++) { t.lo[k] = std::max(b.lo[k], in[i].wbox[k]); t.hi[k] = std::min(b.hi[k], in[i].wbox[3 + k]); }
            bool ok = true;
            for (int k = 0; k < 3; k++) ok = ok && t.lo[k] <= t.hi[k];
            if (ok) b = t;
        }
        // pad: relative to extent and to coordinate magnitude so FP32 slabs stay conservative
        double ext = std::max(b.hi[0] - b.lo[0], std::max(b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]));
        double mag = 0.0;
        for (int k = 0; k < 3; k++) mag = std::max(mag, std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k])));
        double pad = 1e-4 * ext + 4e-6 * mag + 1e-3;
        for (int k = 0; k < 3; k++) { b.lo[k] -= pad; b.hi[k] += pad; }
        all[i] = b;
        scene.grow(b);
    }
    // global leaves: the largest boxes covering a large part of the scene
    std::vector<char> is_global(n_all, 0);
    {
        std::vector<int> cand;
        const double thr = global_frac * scene.area();
        for (int i = 0; i < n_all; i++)
            if (global_frac > 0.0 && all[i].area() >= thr) cand.push_back(i);
        std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return all[a].area() > all[b].area(); });
        if ((int)cand.size() > max_global) cand.resize(std::max(0, max_global));
        for (int i : cand) is_global[i] = 1;
        for (int i = 0; i < n_all; i++)
            if (is_global[i]) {
                out.globals.push_back(in[i].leaf);
                out.global_sphere.insert(out.global_sphere.end(), in[i].sphere, in[i].sphere + 4);
            }
    }
    std::vector<int> keep;
    for (int i = 0; i < n_all; i++) if (!is_global[i]) keep.push_back(i);
    const int n = (int)keep.size();
    out.leaf_count = n;
    Builder B;
    B.boxes.resize(n);
    B.cent.resize(3 * (size_t)n);
    B.idx.resize(n);
    Box ub;
    for (int j = 0; j < n; j++) {
        B.boxes[j] = all[keep[j]];
        ub.grow(B.boxes[j]);
        for (int k = 0; k < 3; k++) B.cent[3 * j + k] = 0.5 * (B.boxes[j].lo[k] + B.boxes[j].hi[k]);
        B.idx[j] = j;
    }
    if (n > 0) {
        // the largest ball about the centre of the hierarchy's box that no leaf box reaches: a ray
        // segment with both ends inside it cannot hit a hierarchy leaf
        double c[3], r2 = std::numeric_limits<double>::infinity();
        for (int k = 0; k < 3; k++) c[k] = 0.5 * (ub.lo[k] + ub.hi[k]);
        for (int j = 0; j < n; j++) {
            double d2 = 0.0;
            for (int k = 0; k < 3; k++) {
                const double e = std::max(B.boxes[j].lo[k] - c[k], std::max(0.0, c[k] - B.boxes[j].hi[k]));
                d2 += e * e;
            }
            r2 = std::min(r2, d2);
        }
        const double r = std::sqrt(r2) * (1.0 - 1e-5) - 1.0;   // 1 mm and a relative margin for FP32 rays
        if (r > 0.0) {
            out.cull[0] = (float)c[0]; out.cull[1] = (float)c[1]; out.cull[2] = (float)c[2];
            out.cull[3] = (float)(r * r);
        }
    }
    if (n == 0) return 0;
    B.nodes.reserve(2 * (size_t)n);
    int root2 = B.build(0, n, 0);
    // reorder leaves
    out.leaves.resize(n);
    out.leaf_sphere.resize(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
        out.leaves[i] = in[keep[B.idx[i]]].leaf;
        for (int k = 0; k < 4; k++) out.leaf_sphere[4 * (size_t)i + k] = in[keep[B.idx[i]]].sphere[k];
    }

    // collapse to 4-wide. Each BVH2 inner node becomes one BVH4 node whose children are
    // the up-to-4 descendants obtained by opening the largest inner child.
    struct Item { int n2; int n4; };
    std::vector<Item> work;
    auto leaf_child = [&](const Node2& nd) { return -(1 + ((nd.first << 3) | (std::max(1, nd.count) - 1))); };
    // a root that is a leaf is wrapped in one BVH4 node with a single child
    out.nodes.push_back(phx_bvh4_node());
    std::memset(&out.nodes[0], 0, sizeof(phx_bvh4_node));
    work.push_back({ root2, 0 });
    while (!work.empty()) {
        Item it = work.back(); work.pop_back();
        const Node2& nd = B.nodes[it.n2];
        int kids[4]; int nk = 0;
        if (is_leaf(nd)) { kids[nk++] = it.n2; }
        else {
            kids[nk++] = nd.left; kids[nk++] = nd.right;
            while (nk < 4) {
                int best = -1; double ba = -1.0;
                for (int k = 0; k < nk; k++) {
                    const Node2& c = B.nodes[kids[k]];
                    if (!is_leaf(c) && c.box.area() > ba) { ba = c.box.area(); best = k; }
                }
                if (best < 0) break;
                const Node2& c = B.nodes[kids[best]];
                kids[best] = c.left;
                kids[nk++] = c.right;
            }
        }
        phx_bvh4_node& o4 = out.nodes[it.n4];
        for (int c = 0; c < 4; c++) {
            if (c >= nk) { set_empty(out.nodes[it.n4], c); continue; }
            const Node2& cn = B.nodes[kids[c]];
            if (is_leaf(cn)) {
                if (cn.count > 8) return -1;   // leaf ranges hold at most 8
                set_child(out.nodes[it.n4], c, cn.box, leaf_child(cn));
            } else {
                int idx4 = (int)out.nodes.size();
                out.nodes.push_back(phx_bvh4_node());
                std::memset(&out.nodes.back(), 0, sizeof(phx_bvh4_node));
                set_child(out.nodes[it.n4], c, cn.box, idx4);
                work.push_back({ kids[c], idx4 });
            }
        }
        (void)o4;
    }
    // depth for the traversal stack bound
    std::vector<int> depth(out.nodes.size(), 0);
    int maxd = 0;
    for (size_t i = 0; i < out.nodes.size(); i++)
        for (int c = 0; c < 4; c++) {
            int ch = out.nodes[i].child[c];
            if (ch > 0) { depth[ch] = depth[i] + 1; maxd = std::max(maxd, depth[ch]); }
        }
    out.max_depth = maxd;
    return 0;
}
