/*
 * speedball_scene.h — host-side scene build helpers of libspeedball_cuda.so.
 *
 * The reference builds each BLAS on the CPU with three-mesh-bvh
 * (new MeshBVH(geometry, { targetLeafSize: 8 }), spectral_scene.js:951;
 * three-mesh-bvh 0.9.14, not vendored) and re-flattens it into the threaded
 * 8 x u32 node layout (flattenBVHRoot, spectral_scene.js:658-721). This
 * builder produces that layout directly: top-down, split on the longest axis
 * of the triangle-centroid bounds at its centre (three-mesh-bvh's default
 * CENTER strategy, restated from its published description), pre-order with
 * the left child at i+1 and miss = first node after the subtree. Node bounds
 * are the exact min/max of the node's triangle vertices. Tree topology parity
 * with three-mesh-bvh itself is unpinned.
 */
#ifndef SPEEDBALL_SCENE_H
#define SPEEDBALL_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Build one local-space BLAS.
 *   pos3:      vertCount x 3 floats
 *   index3:    triCount x 3 vertex indices
 *   maxLeaf:   leaf size (1..255; the pool packs counts into 8 bits)
 *   nodesOut:  capacity 2*triCount nodes x 8 u32; miss links and leaf
 *              triangle offsets are relative to this BLAS (the pool assembly
 *              adds its node and triangle bases, spectral_scene.js:1225-1234)
 *   triOrder:  triCount entries: source triangle at each BVH position
 * Returns the node count, or 0 on invalid input. */
uint32_t sbh_build_blas(const float* pos3, uint32_t vertCount, const uint32_t* index3, uint32_t triCount,
                        uint32_t maxLeaf, uint32_t* nodesOut, uint32_t* triOrder);

#ifdef __cplusplus
}
#endif
#endif /* SPEEDBALL_SCENE_H */
