// sb_flat.h — the scene BVH (derived): one binary tree over every active
// instance's triangles with world-space bounds, in child-pair nodes.
//
// Node (4 x uint4, 64 bytes): q0 = child0 (minx, maxx, miny, maxy),
// q1 = child1 (same), q2 = (child0 minz, maxz, child1 minz, maxz),
// q3 = (entry0, entry1, 0, 0). Entry: a pair-node index (< 2^24), or
// ENTRY_LEAF | count << 24 | first — `count` items from `first` in the item
// array, each item (triangle, instance slot) — or ENTRY_NONE.
//
// Item bounds are the world-space bounds of the triangle under the instance
// transform, widened by a relative margin so that every hit of the reference's
// local-space test lies inside them; the hit tests themselves run in local
// space on the instance's local ray.
#pragma once
#include <stdint.h>

#include <vector>

namespace sb {
namespace flat {

constexpr uint32_t ENTRY_NONE = 0xFFFFFFFFu;
constexpr uint32_t ENTRY_LEAF = 0x80000000u;

struct Tree {
    std::vector<uint32_t> nodes;  // 16 words per pair node
    std::vector<uint32_t> items;  // (triangle, slot) per item, in leaf order
    uint32_t root = ENTRY_NONE;   // entry of the root
    uint32_t depth = 0;           // deepest leaf below the root
    float rootBox[6] = {0, 0, 0, 0, 0, 0};
};

// boxes: 6 floats per item (lo xyz, hi xyz). Returns false when the item count
// does not fit the entry encoding.
bool build(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, Tree& out);

// The same items as an 8-wide tree with 8-bit child boxes (80-byte nodes,
// 20 words), collapsed from the binary SAH tree built with leaves of at most
// WIDE_LEAF_MAX items:
//   w0..w2  node origin p (f32)          w3  ex | ey<<8 | ez<<16 | imask<<24
//   w4      first interior child node    w5  first item of the leaf children
//   w6..w7  meta byte per slot 0..7      w8..w19  qlo x,y,z then qhi x,y,z,
//                                                 two words (slots 0-3, 4-7) each
// Child box on axis a: p + q * 2^(e_a - 127), q rounded outward. imask bit s:
// slot s holds an interior child, the (popcount of imask below s)-th node
// from w4. meta: 0 empty; interior (1 << 5) | (24 + s); leaf ((1 << cnt) - 1)
// << 5 | its first item's offset from w5 (0..23). Slot bits (x, y, z) place a
// child toward +x, +y, +z of the node centre, so visiting slots in increasing
// order of (slot XOR ray-octant) goes roughly near to far.
constexpr uint32_t WIDE_WORDS = 20;
constexpr uint32_t WIDE_LEAF_MAX = 3;

struct WideTree {
    std::vector<uint32_t> nodes;  // WIDE_WORDS per node, root first
    std::vector<uint32_t> items;  // (triangle, slot) per item
    uint32_t depth = 0;           // deepest node level below the root
};

bool build_wide(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, WideTree& out);

}  // namespace flat
}  // namespace sb
