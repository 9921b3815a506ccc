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
    uint32_t maxLeaf = 4;
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
        if (n <= maxLeaf && (bestAxis < 0 || best + nb.area() >= leafCost)) return hi;
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

namespace sb {
namespace flat {

namespace {

// Outward-rounded 8-bit grid of one axis: lo + q * 2^e covers [lo, hi] for q
// in 0..255. Returns the biased exponent (e + 127) stored in the node.
int axis_exponent(float lo, float hi) {
    double extent = (double)hi - (double)lo;
    int e = -126;
    if (extent > 0.0) {
        e = (int)std::ceil(std::log2(extent / 255.0));
        while (std::ldexp(255.0, e) < extent) ++e;
        e = std::max(e, -126);
    }
    return std::min(e, 127) + 127;
}

}  // namespace

bool build_wide(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, WideTree& out) {
    out = WideTree{};
    if (n == 0) return true;
    if (n >= (1u << 24)) return false;
    Builder B;
    B.maxLeaf = WIDE_LEAF_MAX;
    B.boxes = boxes;
    B.cen.resize(3 * (size_t)n);
    B.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) B.cen[3 * (size_t)i + a] = 0.5f * (boxes[6 * (size_t)i + a] + boxes[6 * (size_t)i + 3 + a]);
        B.order[i] = i;
    }
    B.build(n);
    for (size_t v = 0; v < B.count.size(); ++v) {
        if (B.count[v] == 0) continue;
        std::stable_sort(B.order.begin() + B.first[v], B.order.begin() + B.first[v] + B.count[v],
                         [&](uint32_t a, uint32_t b) { return itemSlot[a] < itemSlot[b]; });
    }

    struct Task { uint32_t v, w, depth; };
    std::vector<Task> queue{{0, 0, 0}};
    out.nodes.assign(WIDE_WORDS, 0u);
    uint32_t maxDepth = 0;
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        const Task t = queue[qi];
        maxDepth = std::max(maxDepth, t.depth);
        // children: open the largest interior child until eight (a leaf root is its own child)
        std::vector<uint32_t> kids;
        if (B.count[t.v]) kids.push_back(t.v);
        else { kids.push_back(B.left[t.v]); kids.push_back(B.right[t.v]); }
        while (kids.size() < 8) {
            int best = -1;
            float bestArea = -1.0f;
            for (size_t k = 0; k < kids.size(); ++k)
                if (B.count[kids[k]] == 0 && B.nodeBox[kids[k]].area() > bestArea) {
                    bestArea = B.nodeBox[kids[k]].area();
                    best = (int)k;
                }
            if (best < 0) break;
            uint32_t v = kids[best];
            kids[best] = B.left[v];
            kids.push_back(B.right[v]);
        }
        // slots by octant: slot bit a set = the child lies toward +a of the node centre
        Box nb;
        for (uint32_t k : kids) nb.grow(B.nodeBox[k]);
        float ctr[3];
        for (int a = 0; a < 3; ++a) ctr[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
        struct Cand { float cost; int kid, slot; };
        std::vector<Cand> cands;
        for (size_t k = 0; k < kids.size(); ++k) {
            const Box& b = B.nodeBox[kids[k]];
            for (int s = 0; s < 8; ++s) {
                float c = 0.0f;
                for (int a = 0; a < 3; ++a) {
                    float d = 0.5f * (b.lo[a] + b.hi[a]) - ctr[a];
                    c += (s >> a & 1) ? -d : d;
                }
                cands.push_back({c, (int)k, s});
            }
        }
        std::stable_sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.cost < y.cost; });
        int slotKid[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        std::vector<int> kidSlot(kids.size(), -1);
        for (const Cand& c : cands)
            if (slotKid[c.slot] < 0 && kidSlot[c.kid] < 0) {
                slotKid[c.slot] = c.kid;
                kidSlot[c.kid] = c.slot;
            }
        // header, children and items
        uint32_t* w = out.nodes.data() + (size_t)t.w * WIDE_WORDS;
        int ex[3];
        for (int a = 0; a < 3; ++a) ex[a] = axis_exponent(nb.lo[a], nb.hi[a]);
        std::memcpy(w + 0, &nb.lo[0], 4);
        std::memcpy(w + 1, &nb.lo[1], 4);
        std::memcpy(w + 2, &nb.lo[2], 4);
        uint32_t imask = 0;
        const uint32_t childBase = (uint32_t)(out.nodes.size() / WIDE_WORDS);
        const uint32_t itemBase = (uint32_t)(out.items.size() / 2);
        uint32_t itemOff = 0;
        uint8_t meta[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint8_t q[6][8];
        for (int s = 0; s < 8; ++s) {
            for (int a = 0; a < 3; ++a) { q[a][s] = 255; q[3 + a][s] = 0; }  // empty slots
            if (slotKid[s] < 0) continue;
            const uint32_t v = kids[slotKid[s]];
            const Box& b = B.nodeBox[v];
            for (int a = 0; a < 3; ++a) {
                const double sc = std::ldexp(1.0, ex[a] - 127);
                double lo = std::floor(((double)b.lo[a] - (double)nb.lo[a]) / sc);
                double hi = std::ceil(((double)b.hi[a] - (double)nb.lo[a]) / sc);
                q[a][s] = (uint8_t)std::min(255.0, std::max(0.0, lo));
                q[3 + a][s] = (uint8_t)std::min(255.0, std::max(0.0, hi));
            }
            if (B.count[v] == 0) {
                imask |= 1u << s;
                meta[s] = (uint8_t)((1u << 5) | (24u + s));
                queue.push_back({v, 0, t.depth + 1});  // node index assigned below, in slot order
            } else {
                const uint32_t cnt = B.count[v];
                meta[s] = (uint8_t)((((1u << cnt) - 1u) << 5) | itemOff);
                for (uint32_t k = 0; k < cnt; ++k) {
                    out.items.push_back(itemTri[B.order[B.first[v] + k]]);
                    out.items.push_back(itemSlot[B.order[B.first[v] + k]]);
                }
                itemOff += cnt;
            }
        }
        // interior children get consecutive node indices in slot order
        uint32_t next = childBase;
        for (size_t k = queue.size() - __builtin_popcount(imask); k < queue.size(); ++k) queue[k].w = next++;
        out.nodes.resize((size_t)next * WIDE_WORDS, 0u);
        w = out.nodes.data() + (size_t)t.w * WIDE_WORDS;
        w[3] = (uint32_t)ex[0] | (uint32_t)ex[1] << 8 | (uint32_t)ex[2] << 16 | imask << 24;
        w[4] = childBase;
        w[5] = itemBase;
        w[6] = meta[0] | meta[1] << 8 | meta[2] << 16 | (uint32_t)meta[3] << 24;
        w[7] = meta[4] | meta[5] << 8 | meta[6] << 16 | (uint32_t)meta[7] << 24;
        for (int r = 0; r < 6; ++r) {
            w[8 + 2 * r] = q[r][0] | q[r][1] << 8 | q[r][2] << 16 | (uint32_t)q[r][3] << 24;
            w[9 + 2 * r] = q[r][4] | q[r][5] << 8 | q[r][6] << 16 | (uint32_t)q[r][7] << 24;
        }
    }
    out.depth = maxDepth;
    return true;
}

}  // namespace flat
}  // namespace sb
