// sb_host_bvh.cpp — host BLAS builder emitting the reference's threaded node
// layout (see include/speedball_scene.h for the contract).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/speedball_scene.h"

namespace {

struct Box {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    void add(const float* p) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], p[a]);
            mx[a] = std::max(mx[a], p[a]);
        }
    }
};

struct Builder {
    const float* pos;
    const uint32_t* idx;
    uint32_t maxLeaf;
    std::vector<uint32_t> order;      // triangle ids in BVH order
    std::vector<float> centroid;      // 3 per triangle: centre of its bounds
    uint32_t* nodes;
    uint32_t nodeCount = 0;

    void tri_box(uint32_t t, Box& b) const {
        for (int k = 0; k < 3; ++k) b.add(pos + (size_t)idx[(size_t)t * 3 + k] * 3);
    }

    // Iterative pre-order build over [lo, hi) of `order`.
    void build(uint32_t n) {
        struct Item { uint32_t lo, hi, node, stage; };
        std::vector<Item> st;
        st.push_back({0, n, alloc(), 0});
        while (!st.empty()) {
            Item& it = st.back();
            if (it.stage == 1) {
                // left subtree done: right child starts at the current end
                it.stage = 2;
                uint32_t lo = it.lo, hi = it.hi, mid = split_of(it.node);
                uint32_t right = alloc();
                st.push_back({mid, hi, right, 0});
                (void)lo;
                continue;
            }
            if (it.stage == 2) {
                nodes[(size_t)it.node * 8 + 6] = nodeCount;  // miss = first node after the subtree
                st.pop_back();
                continue;
            }
            uint32_t lo = it.lo, hi = it.hi, node = it.node;
            Box b, c;
            for (uint32_t i = lo; i < hi; ++i) {
                tri_box(order[i], b);
                c.add(&centroid[(size_t)order[i] * 3]);
            }
            uint32_t* nd = nodes + (size_t)node * 8;
            for (int a = 0; a < 3; ++a) {
                std::memcpy(&nd[a], &b.mn[a], 4);
                std::memcpy(&nd[3 + a], &b.mx[a], 4);
            }
            uint32_t count = hi - lo;
            if (count <= maxLeaf) {
                nd[6] = nodeCount;  // leaf: miss = next slot
                nd[7] = (count << 24) | lo;
                st.pop_back();
                continue;
            }
            int axis = 0;
            float ext[3];
            for (int a = 0; a < 3; ++a) ext[a] = c.mx[a] - c.mn[a];
            if (ext[1] > ext[axis]) axis = 1;
            if (ext[2] > ext[axis]) axis = 2;
            uint32_t mid;
            if (ext[axis] > 0.0f) {
                float pivot = (c.mn[axis] + c.mx[axis]) * 0.5f;
                auto it2 = std::partition(order.begin() + lo, order.begin() + hi,
                                          [&](uint32_t t) { return centroid[(size_t)t * 3 + axis] < pivot; });
                mid = (uint32_t)(it2 - order.begin());
            } else {
                mid = lo;
            }
            if (mid == lo || mid == hi) mid = lo + count / 2;  // degenerate split: halve by index
            nd[7] = 0xFFFFFFFFu;
            nd[6] = mid;  // stash the split until the left subtree is built
            it.stage = 1;
            uint32_t left = alloc();
            st.push_back({lo, mid, left, 0});
        }
    }
    uint32_t alloc() { return nodeCount++; }
    uint32_t split_of(uint32_t node) const { return nodes[(size_t)node * 8 + 6]; }
};

}  // namespace

extern "C" uint32_t sbh_build_blas(const float* pos3, uint32_t vertCount, const uint32_t* index3, uint32_t triCount,
                                   uint32_t maxLeaf, uint32_t* nodesOut, uint32_t* triOrder) {
    if (!pos3 || !index3 || !nodesOut || !triOrder || triCount == 0 || maxLeaf == 0 || maxLeaf > 255) return 0;
    for (size_t i = 0; i < (size_t)triCount * 3; ++i)
        if (index3[i] >= vertCount) return 0;
    Builder B;
    B.pos = pos3;
    B.idx = index3;
    B.maxLeaf = maxLeaf;
    B.nodes = nodesOut;
    B.order.resize(triCount);
    B.centroid.resize((size_t)triCount * 3);
    for (uint32_t t = 0; t < triCount; ++t) {
        B.order[t] = t;
        Box b;
        B.tri_box(t, b);
        for (int a = 0; a < 3; ++a) B.centroid[(size_t)t * 3 + a] = b.mn[a] + (b.mx[a] - b.mn[a]) * 0.5f;
    }
    B.build(triCount);
    std::memcpy(triOrder, B.order.data(), (size_t)triCount * 4);
    return B.nodeCount;
}
