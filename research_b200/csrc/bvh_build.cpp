// bvh_build.cpp — host binned-SAH BVH2 builder.
//
// Replaces the driver-built BLAS/TLAS of the reference
// (AccelStructure.cpp:98-330, PREFER_FAST_TRACE). Builds one binary tree
// over world-space triangles (32 centroid bins per axis, surface-area cost,
// leaves of at most 8 triangles, depth capped at 60 so a 64-entry traversal
// stack always suffices), then lays it out for the GPU: every inner node
// stores the boxes of both children, inner nodes in depth-first order.
// Large subtrees are built on separate threads. The same tree is also laid
// out 4-wide: a 4-wide node's children are a binary node's frontier of up to
// four nodes, grown by opening the inner frontier node of largest surface
// area (the leaves are the binary tree's leaves).

#include "rr_bvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>

namespace rr {
namespace {

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    float area() const {
        if (!(hi[0] >= lo[0])) return 0.0f;
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node {
    Box box;
    int32_t left = -1, right = -1;  // binary children; -1 = leaf
    uint32_t first = 0, count = 0;
};

constexpr int kBins = 32;
constexpr uint32_t kMaxLeaf = 8;
constexpr uint32_t kMaxDepth = 60;

struct Builder {
    const std::vector<Box>& boxes;
    const std::vector<float>& cent;  // 3 per tri
    std::vector<uint32_t>& order;
    std::vector<Node>& nodes;
    std::atomic<uint32_t> next{1};
    std::atomic<uint32_t> depth_max{0};

    void make_leaf(uint32_t idx, uint32_t first, uint32_t count) {
        nodes[idx].left = nodes[idx].right = -1;
        nodes[idx].first = first; nodes[idx].count = count;
    }

    void build(uint32_t idx, uint32_t first, uint32_t count, uint32_t depth) {
        uint32_t dm = depth_max.load();
        while (depth > dm && !depth_max.compare_exchange_weak(dm, depth)) {}
        Box box, cbox;
        for (uint32_t i = first; i < first + count; ++i) {
            box.grow(boxes[order[i]]);
            cbox.grow(&cent[3 * order[i]]);
        }
        nodes[idx].box = box;
        if (count <= 1 || depth >= kMaxDepth) { make_leaf(idx, first, count); return; }

        // Binned SAH over the three axes.
        float best_cost = INFINITY;
        int best_axis = -1, best_split = 0;
        for (int a = 0; a < 3; ++a) {
            const float ext = cbox.hi[a] - cbox.lo[a];
            if (!(ext > 0.0f)) continue;
            const float scale = float(kBins) * (1.0f - 1e-6f) / ext;
            uint32_t cnt[kBins] = {};
            Box bb[kBins];
            for (uint32_t i = first; i < first + count; ++i) {
                const uint32_t t = order[i];
                int b = int((cent[3 * t + a] - cbox.lo[a]) * scale);
                b = std::min(std::max(b, 0), kBins - 1);
                cnt[b]++;
                bb[b].grow(boxes[t]);
            }
            float right_area[kBins];
            uint32_t right_cnt[kBins];
            Box acc; uint32_t c = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bb[b]); c += cnt[b];
                right_area[b] = acc.area(); right_cnt[b] = c;
            }
            acc = Box(); c = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bb[b]); c += cnt[b];
                if (c == 0 || right_cnt[b + 1] == 0) continue;
                const float cost = acc.area() * float(c) + right_area[b + 1] * float(right_cnt[b + 1]);
                if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = b + 1; }
            }
        }
        const float leaf_cost = box.area() * float(count);
        const float split_cost = box.area() + best_cost;  // one node visit + children
        uint32_t mid;
        if (best_axis < 0) {
            if (count <= kMaxLeaf) { make_leaf(idx, first, count); return; }
            mid = first + count / 2;  // all centroids equal: split the list
        } else {
            if (count <= kMaxLeaf && leaf_cost <= split_cost) { make_leaf(idx, first, count); return; }
            const int a = best_axis;
            const float ext = cbox.hi[a] - cbox.lo[a];
            const float scale = float(kBins) * (1.0f - 1e-6f) / ext;
            auto it = std::partition(order.begin() + first, order.begin() + first + count, [&](uint32_t t) {
                int b = int((cent[3 * t + a] - cbox.lo[a]) * scale);
                b = std::min(std::max(b, 0), kBins - 1);
                return b < best_split;
            });
            mid = uint32_t(it - order.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        }
        const uint32_t l = next.fetch_add(2);
        const uint32_t r = l + 1;
        nodes[idx].left = int32_t(l);
        nodes[idx].right = int32_t(r);
        const uint32_t nl = mid - first, nr = first + count - mid;
        if (depth < 8 && count > 50000) {
            auto fut = std::async(std::launch::async, [=]() { build(l, first, nl, depth + 1); });
            build(r, mid, nr, depth + 1);
            fut.get();
        } else {
            build(l, first, nl, depth + 1);
            build(r, mid, nr, depth + 1);
        }
    }
};

inline float4 mk4(float x, float y, float z, float w) { float4 v; v.x = x; v.y = y; v.z = z; v.w = w; return v; }
inline float i2f(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }

// 4-wide layout (8 float4 per node): lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of
// children 0..3, then their references (>= 0 a node, < 0 a leaf starting at
// triangle ~ref) and their triangle counts. An unused child slot gets a
// point box at 1e30 on every axis, which no ray reaches within its tmax.
struct Wide4 {
    const std::vector<Node>& nodes;
    std::vector<float4>& out;
    int32_t emit(const std::vector<uint32_t>& kids) {
        const int32_t idx = int32_t(out.size() / 8);
        out.resize(out.size() + 8);
        float lo[3][4], hi[3][4];
        int32_t ref[4] = {0, 0, 0, 0}, cnt[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k)
            for (int a = 0; a < 3; ++a) lo[a][k] = hi[a][k] = 1e30f;
        for (size_t k = 0; k < kids.size(); ++k) {
            const Node& c = nodes[kids[k]];
            for (int a = 0; a < 3; ++a) { lo[a][k] = c.box.lo[a]; hi[a][k] = c.box.hi[a]; }
            if (c.left < 0) { ref[k] = ~int32_t(c.first); cnt[k] = int32_t(c.count); }
            else ref[k] = emit(frontier(kids[k]));
        }
        float4* q = &out[size_t(idx) * 8];
        for (int a = 0; a < 3; ++a) {
            q[2 * a] = mk4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
            q[2 * a + 1] = mk4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
        }
        q[6] = mk4(i2f(ref[0]), i2f(ref[1]), i2f(ref[2]), i2f(ref[3]));
        q[7] = mk4(i2f(cnt[0]), i2f(cnt[1]), i2f(cnt[2]), i2f(cnt[3]));
        return idx;
    }
    // the up-to-four-node frontier below inner binary node b
    std::vector<uint32_t> frontier(uint32_t b) const {
        std::vector<uint32_t> kids{uint32_t(nodes[b].left), uint32_t(nodes[b].right)};
        while (kids.size() < 4) {
            int best = -1;
            float best_area = -1.0f;
            for (size_t k = 0; k < kids.size(); ++k) {
                if (nodes[kids[k]].left < 0) continue;
                const float ar = nodes[kids[k]].box.area();
                if (ar > best_area) { best_area = ar; best = int(k); }
            }
            if (best < 0) break;
            const uint32_t c = kids[best];
            kids[best] = uint32_t(nodes[c].left);
            kids.insert(kids.begin() + best + 1, uint32_t(nodes[c].right));
        }
        return kids;
    }
};

} // namespace

BvhBuild build_bvh(const std::vector<float>& tri_world, int /*threads*/) {
    const uint32_t n = uint32_t(tri_world.size() / 9);
    BvhBuild out;
    std::vector<Box> boxes(n);
    std::vector<float> cent(size_t(n) * 3);
    for (uint32_t i = 0; i < n; ++i) {
        Box b;
        b.grow(&tri_world[9 * size_t(i)]);
        b.grow(&tri_world[9 * size_t(i) + 3]);
        b.grow(&tri_world[9 * size_t(i) + 6]);
        boxes[i] = b;
        for (int a = 0; a < 3; ++a) cent[3 * size_t(i) + a] = 0.5f * (b.lo[a] + b.hi[a]);
    }
    out.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) out.order[i] = i;
    std::vector<Node> nodes(std::max<size_t>(1, 2 * size_t(n)));
    Builder B{boxes, cent, out.order, nodes};
    if (n > 0) B.build(0, 0, n, 0);
    else nodes[0].box = Box();
    out.max_depth = B.depth_max.load() + 1;
    {
        Wide4 W{nodes, out.nodes4};
        if (n > 0 && nodes[0].left >= 0) W.emit(W.frontier(0));
        else if (n > 0) W.emit(std::vector<uint32_t>{0u});   // the root is a leaf
        else W.emit(std::vector<uint32_t>{});
    }

    // GPU layout: one GPU node per inner binary node, depth-first, left first.
    auto child_ref = [&](const Node& c, std::vector<int32_t>& gidx, int32_t ci, int32_t& ref, int32_t& cnt) {
        if (c.left < 0) { ref = ~int32_t(c.first); cnt = int32_t(c.count); }
        else { ref = gidx[ci]; cnt = 0; }
    };
    std::vector<int32_t> gidx(nodes.size(), -1);
    std::vector<uint32_t> dfs;
    if (nodes[0].left < 0) {
        // Root is a leaf: one GPU node with the leaf and an empty sibling.
        const Node& r = nodes[0];
        const Box& b = r.box;
        const float lo0 = n ? b.lo[0] : 0.f, hi0 = n ? b.hi[0] : 0.f;
        const float lo1 = n ? b.lo[1] : 0.f, hi1 = n ? b.hi[1] : 0.f;
        const float lo2 = n ? b.lo[2] : 0.f, hi2 = n ? b.hi[2] : 0.f;
        out.nodes.push_back(mk4(lo0, hi0, lo1, hi1));
        out.nodes.push_back(mk4(lo0, hi0, lo1, hi1));
        out.nodes.push_back(mk4(lo2, hi2, lo2, hi2));
        out.nodes.push_back(mk4(i2f(~int32_t(0)), i2f(~int32_t(0)), i2f(int32_t(r.count)), i2f(0)));
        return out;
    }
    // iterative DFS to assign GPU indices
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
        const uint32_t i = stack.back(); stack.pop_back();
        gidx[i] = int32_t(dfs.size());
        dfs.push_back(i);
        const Node& nd = nodes[i];
        if (nodes[nd.right].left >= 0) stack.push_back(uint32_t(nd.right));
        if (nodes[nd.left].left >= 0) stack.push_back(uint32_t(nd.left));
    }
    out.nodes.resize(dfs.size() * 4);
    for (size_t g = 0; g < dfs.size(); ++g) {
        const Node& nd = nodes[dfs[g]];
        const Node& c0 = nodes[nd.left];
        const Node& c1 = nodes[nd.right];
        int32_t r0, r1, k0, k1;
        child_ref(c0, gidx, nd.left, r0, k0);
        child_ref(c1, gidx, nd.right, r1, k1);
        out.nodes[g * 4 + 0] = mk4(c0.box.lo[0], c0.box.hi[0], c0.box.lo[1], c0.box.hi[1]);
        out.nodes[g * 4 + 1] = mk4(c1.box.lo[0], c1.box.hi[0], c1.box.lo[1], c1.box.hi[1]);
        out.nodes[g * 4 + 2] = mk4(c0.box.lo[2], c0.box.hi[2], c1.box.lo[2], c1.box.hi[2]);
        out.nodes[g * 4 + 3] = mk4(i2f(r0), i2f(r1), i2f(k0), i2f(k1));
    }
    return out;
}

} // namespace rr
