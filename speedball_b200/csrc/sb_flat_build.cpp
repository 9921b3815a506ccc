// sb_flat_build.cpp — host builder of the scene BVH: a binned-SAH binary tree
// over (triangle, instance slot) items with world-space bounds, emitted in the
// child-pair layout the traversal reads (sb_flat.h).
//
// This is a derived acceleration structure, built on structural changes only
// (scene upload, instance set, TLAS build), like the reference's CPU-built
// BVHs. The reference's per-instance BLASes and TLAS stay the wire format and
// are still refit and rebuilt bit-exactly; the scene BVH only decides which
// (triangle, instance) pairs a ray tests, and the tests themselves run in the
// instance's local space exactly as the reference's.
#include "sb_flat.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace sb {
namespace flat {

namespace {

constexpr int BINS = 16;
constexpr uint32_t MAX_LEAF = 4;

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    float area() const {
        float d[3];
        for (int a = 0; a < 3; ++a) d[a] = hi[a] - lo[a];
        if (d[0] < 0.f) return 0.f;
        return 2.f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct Builder {
    const float* boxes;  // 6 per item
    std::vector<float> cen;
    std::vector<uint32_t> order;
    std::vector<Box> nodeBox;        // per tree node (interior and leaf)
    std::vector<uint32_t> left, right, first, count;  // count == 0 -> interior

    Box item_box(uint32_t i) const {
        Box b;
        std::memcpy(b.lo, boxes + 6 * (size_t)i, 12);
        std::memcpy(b.hi, boxes + 6 * (size_t)i + 3, 12);
        return b;
    }

    uint32_t make_node() {
        nodeBox.emplace_back();
        left.push_back(0);
        right.push_back(0);
        first.push_back(0);
        count.push_back(0);
        return (uint32_t)nodeBox.size() - 1;
    }

    // Splits [lo, hi) of `order`; returns the split point or hi for a leaf.
    uint32_t split(uint32_t lo, uint32_t hi, const Box& nb) {
        const uint32_t n = hi - lo;
        if (n <= 1) return hi;
        Box cb;
        for (uint32_t k = lo; k < hi; ++k) cb.grow(&cen[3 * (size_t)order[k]]);
        float best = INFINITY;
        int bestAxis = -1, bestBin = 0;
        for (int a = 0; a < 3; ++a) {
            float c0 = cb.lo[a], c1 = cb.hi[a];
            if (!(c1 > c0)) continue;
            const float scale = BINS / (c1 - c0);
            Box bb[BINS];
            uint32_t bc[BINS] = {};
            for (uint32_t k = lo; k < hi; ++k) {
                uint32_t i = order[k];
                int b = std::min(BINS - 1, (int)((cen[3 * (size_t)i + a] - c0) * scale));
                bb[b].grow(item_box(i));
                ++bc[b];
            }
            float la[BINS];
            uint32_t lc[BINS];
            Box L;
            uint32_t ln = 0;
            for (int b = 0; b < BINS - 1; ++b) {
                L.grow(bb[b]);
                ln += bc[b];
                la[b] = L.area();
                lc[b] = ln;
            }
            Box R;
            uint32_t rn = 0;
            for (int b = BINS - 1; b > 0; --b) {
                R.grow(bb[b]);
                rn += bc[b];
                if (lc[b - 1] == 0 || rn == 0) continue;
                float cost = la[b - 1] * lc[b - 1] + R.area() * rn;
                if (cost < best) {
                    best = cost;
                    bestAxis = a;
                    bestBin = b;
                }
            }
        }
        // SAH: traversal step ~ one item test; stop when splitting costs more
        const float leafCost = nb.area() * n;
        if (n <= MAX_LEAF && (bestAxis < 0 || best + nb.area() >= leafCost)) return hi;
        uint32_t mid = lo + n / 2;
        if (bestAxis >= 0) {
            const float c0 = cb.lo[bestAxis], scale = BINS / (cb.hi[bestAxis] - c0);
            auto it = std::partition(order.begin() + lo, order.begin() + hi, [&](uint32_t i) {
                return std::min(BINS - 1, (int)((cen[3 * (size_t)i + bestAxis] - c0) * scale)) < bestBin;
            });
            mid = (uint32_t)(it - order.begin());
        }
        if (mid == lo || mid == hi) {  // coincident centroids: split by index
            mid = lo + n / 2;
        }
        return mid;
    }

    void build(uint32_t n) {
        struct Task { uint32_t lo, hi, node; };
        std::vector<Task> st;
        uint32_t root = make_node();
        st.push_back({0, n, root});
        while (!st.empty()) {
            Task t = st.back();
            st.pop_back();
            Box nb;
            for (uint32_t k = t.lo; k < t.hi; ++k) nb.grow(item_box(order[k]));
            nodeBox[t.node] = nb;
            uint32_t mid = split(t.lo, t.hi, nb);
            if (mid >= t.hi) {
                first[t.node] = t.lo;
                count[t.node] = t.hi - t.lo;
                continue;
            }
            uint32_t l = make_node(), r = make_node();
            left[t.node] = l;
            right[t.node] = r;
            st.push_back({mid, t.hi, r});
            st.push_back({t.lo, mid, l});
        }
    }
};

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace

bool build(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, Tree& out) {
    out = Tree{};
    if (n == 0) {
        out.root = ENTRY_NONE;
        return true;
    }
    if (n >= (1u << 24)) return false;
    Builder B;
    B.boxes = boxes;
    B.cen.resize(3 * (size_t)n);
    B.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) B.cen[3 * (size_t)i + a] = 0.5f * (boxes[6 * (size_t)i + a] + boxes[6 * (size_t)i + 3 + a]);
        B.order[i] = i;
    }
    B.build(n);

    // leaves: items ordered by slot, so consecutive tests reuse the local ray
    for (size_t v = 0; v < B.count.size(); ++v) {
        if (B.count[v] == 0) continue;
        std::stable_sort(B.order.begin() + B.first[v], B.order.begin() + B.first[v] + B.count[v],
                         [&](uint32_t a, uint32_t b) { return itemSlot[a] < itemSlot[b]; });
    }
    out.items.resize(2 * (size_t)n);
    for (uint32_t k = 0; k < n; ++k) {
        out.items[2 * (size_t)k] = itemTri[B.order[k]];
        out.items[2 * (size_t)k + 1] = itemSlot[B.order[k]];
    }

    // pair nodes: one per interior tree node, numbered in pre-order
    const size_t total = B.nodeBox.size();
    std::vector<uint32_t> pairIndex(total, ENTRY_NONE);
    std::vector<uint32_t> depth(total, 0);
    uint32_t pairs = 0, maxDepth = 0;
    {
        std::vector<uint32_t> st{0};
        while (!st.empty()) {
            uint32_t v = st.back();
            st.pop_back();
            maxDepth = std::max(maxDepth, depth[v]);
            if (B.count[v]) continue;
            pairIndex[v] = pairs++;
            depth[B.left[v]] = depth[B.right[v]] = depth[v] + 1;
            st.push_back(B.right[v]);
            st.push_back(B.left[v]);
        }
    }
    auto entry = [&](uint32_t v) -> uint32_t {
        if (B.count[v] == 0) return pairIndex[v];
        return ENTRY_LEAF | (B.count[v] << 24) | B.first[v];
    };
    out.nodes.assign(16 * (size_t)pairs, 0u);
    for (size_t v = 0; v < total; ++v) {
        if (B.count[v]) continue;
        uint32_t* q = out.nodes.data() + 16 * (size_t)pairIndex[v];
        const Box& a = B.nodeBox[B.left[v]];
        const Box& b = B.nodeBox[B.right[v]];
        q[0] = fbits(a.lo[0]); q[1] = fbits(a.hi[0]); q[2] = fbits(a.lo[1]); q[3] = fbits(a.hi[1]);
        q[4] = fbits(b.lo[0]); q[5] = fbits(b.hi[0]); q[6] = fbits(b.lo[1]); q[7] = fbits(b.hi[1]);
        q[8] = fbits(a.lo[2]); q[9] = fbits(a.hi[2]); q[10] = fbits(b.lo[2]); q[11] = fbits(b.hi[2]);
        q[12] = entry(B.left[v]);
        q[13] = entry(B.right[v]);
    }
    out.root = entry(0);
    out.depth = maxDepth;
    std::memcpy(out.rootBox, B.nodeBox[0].lo, 12);
    std::memcpy(out.rootBox + 3, B.nodeBox[0].hi, 12);
    return true;
}

}  // namespace flat
}  // namespace sb
