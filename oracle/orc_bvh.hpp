// orc_bvh.hpp — the BLAS build of the reference's scene pool, restated:
// `new MeshBVH(geometry, { targetLeafSize: 8, indirect: false })`
// (spectral_scene.js:951) followed by flattenBVHRoot (658-721).
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
//
// MeshBVH is the third-party three-mesh-bvh (peer range >=0.9.11 <0.10.0,
// package.json:69; demo pin 0.9.14, index.html:17), not vendored with the
// reference. Restated from its published build with the default CENTER
// strategy:
//   * per triangle, per axis: centre and half extent of its vertex bounds,
//     computed in double and stored as float32 (a Float32Array);
//   * a node's bounds are the union of (centre - half, centre + half) over its
//     triangles; the centroid bounds are the union of the centres;
//   * a node with count <= the leaf size, or at depth >= 40, is a leaf;
//   * split axis = the longest axis of the centroid bounds (first on ties),
//     position = the middle of the centroid bounds on that axis;
//   * Hoare partition of the range: triangles whose centre is < position go
//     left, the rest right (index triples and bounds swapped in place);
//   * an empty side makes the node a leaf.
// flattenBVHRoot then writes the nodes in pre-order with the left child next
// (idx + 1) and every node's miss = the first index after its subtree, leaves
// as (count << 24) | offset with offsets in triangle units of the permuted index.
// Parity against three-mesh-bvh itself is unpinned (the module is absent); any
// valid BVH gives the same closest hits up to exact-t ties.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

struct MeshBvhBuild {
    const float* pos = nullptr;   // 3 floats per vertex
    uint32_t* index = nullptr;    // 3 per triangle, permuted in place
    uint32_t leafSize = 8;
    uint32_t maxDepth = 40;
    std::vector<float> tb;        // 6 per triangle: (centre, half) per axis
    std::vector<uint32_t> order;  // source triangle id at each position
    std::vector<uint32_t> out;    // 8 u32 per emitted node
    bool overflow = false;        // a leaf above the 8-bit count field

    void triangle_bounds(uint32_t T) {
        tb.assign((size_t)T * 6, 0.0f);
        order.resize(T);
        for (uint32_t t = 0; t < T; ++t) {
            order[t] = t;
            for (int a = 0; a < 3; ++a) {
                double mn = INFINITY, mx = -INFINITY;
                for (int k = 0; k < 3; ++k) {
                    double v = pos[(size_t)index[(size_t)t * 3 + k] * 3 + a];
                    mn = std::min(mn, v);
                    mx = std::max(mx, v);
                }
                double half = (mx - mn) / 2.0;
                tb[(size_t)t * 6 + a * 2] = (float)(mn + half);
                tb[(size_t)t * 6 + a * 2 + 1] = (float)half;
            }
        }
    }

    void bounds(uint32_t off, uint32_t cnt, float box[6], float cbox[6]) const {
        double b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        double c[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = off; i < off + cnt; ++i)
            for (int a = 0; a < 3; ++a) {
                double cen = tb[(size_t)i * 6 + a * 2], h = tb[(size_t)i * 6 + a * 2 + 1];
                b[a] = std::min(b[a], cen - h);
                b[a + 3] = std::max(b[a + 3], cen + h);
                c[a] = std::min(c[a], cen);
                c[a + 3] = std::max(c[a + 3], cen);
            }
        for (int k = 0; k < 6; ++k) {
            box[k] = (float)b[k];
            cbox[k] = (float)c[k];
        }
    }

    void swap_tri(uint32_t i, uint32_t j) {
        for (int k = 0; k < 3; ++k) std::swap(index[(size_t)i * 3 + k], index[(size_t)j * 3 + k]);
        for (int k = 0; k < 6; ++k) std::swap(tb[(size_t)i * 6 + k], tb[(size_t)j * 6 + k]);
        std::swap(order[i], order[j]);
    }

    uint32_t partition(uint32_t off, uint32_t cnt, int axis, double p) {
        int64_t left = off, right = (int64_t)off + cnt - 1;
        for (;;) {
            while (left <= right && tb[(size_t)left * 6 + axis * 2] < p) ++left;
            while (left <= right && tb[(size_t)right * 6 + axis * 2] >= p) --right;
            if (left < right) {
                swap_tri((uint32_t)left, (uint32_t)right);
                ++left;
                --right;
            } else {
                return (uint32_t)left;
            }
        }
    }

    // Emits the subtree of [off, off + cnt) in pre-order.
    void emit(uint32_t off, uint32_t cnt, uint32_t depth) {
        struct Frame { uint32_t off, cnt, depth, node, split, stage; };
        std::vector<Frame> st;
        st.push_back({off, cnt, depth, 0, 0, 0});
        while (!st.empty()) {
            Frame& f = st.back();
            if (f.stage == 1) {  // left subtree written: the right child follows
                f.stage = 2;
                Frame r{f.split, f.off + f.cnt - f.split, f.depth + 1, 0, 0, 0};
                st.push_back(r);
                continue;
            }
            if (f.stage == 2) {
                out[(size_t)f.node * 8 + 6] = (uint32_t)(out.size() / 8);
                st.pop_back();
                continue;
            }
            float box[6], cbox[6];
            bounds(f.off, f.cnt, box, cbox);
            f.node = (uint32_t)(out.size() / 8);
            out.resize(out.size() + 8, 0u);
            uint32_t* nd = &out[(size_t)f.node * 8];
            std::memcpy(nd, box, 24);
            bool leaf = f.cnt <= leafSize || f.depth >= maxDepth;
            uint32_t split = 0;
            if (!leaf) {
                int axis = -1;
                double best = -INFINITY;
                for (int a = 0; a < 3; ++a) {
                    double d = (double)cbox[a + 3] - (double)cbox[a];
                    if (d > best) { best = d; axis = a; }
                }
                double p = ((double)cbox[axis] + (double)cbox[axis + 3]) / 2.0;
                split = partition(f.off, f.cnt, axis, p);
                leaf = split == f.off || split == f.off + f.cnt;
            }
            if (leaf) {
                if (f.cnt > 255u) overflow = true;
                nd[6] = f.node + 1;
                nd[7] = ((f.cnt & 0xFFu) << 24) | (f.off & 0x00FFFFFFu);
                st.pop_back();
                continue;
            }
            nd[7] = 0xFFFFFFFFu;
            f.split = split;
            f.stage = 1;
            Frame l{f.off, split - f.off, f.depth + 1, 0, 0, 0};
            st.push_back(l);
        }
    }
};

// Returns the node count (0 on an empty mesh, an out-of-range index, or a
// leaf larger than the 8-bit count field).
inline uint32_t build_mesh_bvh(const float* pos3, uint32_t vertCount, uint32_t* index3, uint32_t triCount,
                               uint32_t leafSize, std::vector<uint32_t>& nodes, std::vector<uint32_t>& order) {
    if (!triCount || !leafSize || leafSize > 255) return 0;
    for (size_t i = 0; i < (size_t)triCount * 3; ++i)
        if (index3[i] >= vertCount) return 0;
    MeshBvhBuild b;
    b.pos = pos3;
    b.index = index3;
    b.leafSize = leafSize;
    b.triangle_bounds(triCount);
    b.emit(0, triCount, 0);
    if (b.overflow) return 0;
    nodes.swap(b.out);
    order.swap(b.order);
    return (uint32_t)(nodes.size() / 8);
}

}  // namespace orc
