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

}  // namespace flat
}  // namespace sb
