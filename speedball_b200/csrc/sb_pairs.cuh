// sb_pairs.cuh — writers of the derived child-pair nodes (layout in
// sb_internal.cuh), shared by the structural derivation (sb_pairs.cu) and the
// refits (sb_refit.cu), which keep the pair boxes bit-identical to the
// reference nodes they copy.
#pragma once
#include "sb_internal.cuh"

namespace sb {

// Entry for a BLAS child given its reference index and payload word.
__device__ __forceinline__ uint32_t blas_entry(uint32_t idx, uint32_t payload) {
    if (payload == INTERIOR) return idx < PE_BLAS_MAX_NODES ? (PE_BLAS | idx) : PE_NONE;
    return (payload >> 24) ? payload : PE_NONE;  // an empty leaf holds nothing to test
}

// Entry for a TLAS child given its index and payload (cnt << 24) | slot.
__device__ __forceinline__ uint32_t tlas_entry(uint32_t idx, uint32_t payload) {
    uint32_t cnt = payload >> 24, slot = payload & 0x00FFFFFFu;
    if (cnt == 0u) return idx < PE_TLEAF ? idx : PE_NONE;
    return (slot < PE_TLAS_MAX_SLOTS && cnt < 1024u) ? (PE_TLEAF | (cnt << 12) | slot) : PE_NONE;
}

// Boxes in the reference word order (minx, miny, minz, maxx, maxy, maxz).
__device__ __forceinline__ void store_pair_boxes(uint4* p, const uint32_t b0[6], const uint32_t b1[6]) {
    p[0] = make_uint4(b0[0], b0[3], b0[1], b0[4]);
    p[1] = make_uint4(b1[0], b1[3], b1[1], b1[4]);
    p[2] = make_uint4(b0[2], b0[5], b1[2], b1[5]);
}

__device__ __forceinline__ void store_pair(uint4* p, const uint32_t b0[6], const uint32_t b1[6], uint32_t e0,
                                           uint32_t e1) {
    store_pair_boxes(p, b0, b1);
    p[3] = make_uint4(e0, e1, 0u, 0u);
}

}  // namespace sb
