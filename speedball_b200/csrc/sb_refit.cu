// sb_refit.cu — the refit and TLAS lanes on the GPU:
//   * BLAS refit (refitFlatBlasRange, gi_refit.js:34-165): exact leaf min/max in
//     the reference's visiting order, interiors as the JS Math.min/max union of
//     (i+1, miss(i+1)); run bottom-up in parallel with arrival counters, fused
//     with the re-gather of the pre-gathered triangles of the deformed leaves.
//   * per-instance transform math (computeDynamic, spectral_scene.js:1262-1294)
//     in FP64 with every operation separately rounded.
//   * TLAS build (buildTlasRecords, spectral_scene.js:973-1003): one CTA, level
//     by level; each level stable-sorts every interior segment by its FP64
//     centroid on the longest axis (a bitonic sort on (segment, key, position),
//     which equals a stable sort) and splits at the index midpoint.
//   * TLAS refit (refitFlatTlasRange, gi_refit.js:245-292): one CTA, deepest
//     level first.
// min/max are exact, so all bounds are bit-identical to the reference walk.
#include "sb_kernels.cuh"
#include "sb_pairs.cuh"

namespace sb {

constexpr uint32_t NONE = 0xFFFFFFFFu;

__device__ __forceinline__ void bad(uint32_t* gate, uint32_t* err) {
    if (gate) *gate = 0u;
    latch(err, ERR_LAYOUT);
}

// ------------------------------------------------------------- BLAS refit
__global__ void k_refit_reset(uint32_t* parent, uint32_t* arrive, uint32_t root, uint32_t end) {
    uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    parent[i] = NONE;
    arrive[i] = 0u;
}

// The end of node i's subtree as its own miss word states it: miss(i) when it
// lies in (i, end], else the range end (the right spine of the range).
__device__ __forceinline__ uint32_t subtree_end(const uint32_t* nodes, uint32_t i, uint32_t end) {
    const uint32_t miss = nodes[8 * i + 6];
    return (miss > i && miss <= end) ? miss : end;
}

// A range's gate word: 0 = the layout check failed (the refit reports
// SB_ERR_LAYOUT_VIOLATION until the next upload); 1 = valid, and every node's
// own miss word ends its subtree (a leaf: i + 1; an interior node: where its
// right child's subtree ends), so subtrees can be cut out by index range;
// 2 = valid for the reference's refit, which reads only left children's miss
// words (gi_refit.js:96-139), while some other miss word is stale: the range is
// refit node by node without the subtree partition.
//
// Link children to parents and check the layout contract (gi_refit.js:96-139):
// right child = left child's miss, inside (left, end); leaves index inside the
// triangle and vertex pools. A node claimed twice, or an orphan, also fails.
__global__ void k_refit_link(const uint32_t* nodes, const uint32_t* triIndex, const uint32_t* triMaterial,
                             uint32_t triCount, uint32_t vertexCount, uint32_t materialCount, uint32_t* parent,
                             uint32_t root, uint32_t end, uint32_t* gate, uint32_t* err) {
    uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    uint32_t info = nodes[8 * i + 7];
    if (info != INTERIOR) {
        uint32_t off = info & 0x00FFFFFFu, cnt = info >> 24;
        for (uint32_t t = off; t < off + cnt; ++t) {
            if (t >= triCount || triMaterial[t] >= materialCount) { bad(gate, err); return; }
            for (int k = 0; k < 3; ++k)
                if (triIndex[3 * t + k] >= vertexCount) { bad(gate, err); return; }
        }
        if (subtree_end(nodes, i, end) != i + 1u) atomicCAS(gate, 1u, 2u);
        return;
    }
    uint32_t l = i + 1;
    if (l >= end) { bad(gate, err); return; }
    uint32_t r = nodes[8 * l + 6];
    if (!(r > l && r < end)) { bad(gate, err); return; }
    if (atomicCAS(&parent[l], NONE, i) != NONE) bad(gate, err);
    if (atomicCAS(&parent[r], NONE, i) != NONE) bad(gate, err);
    if (subtree_end(nodes, i, end) != subtree_end(nodes, r, end)) atomicCAS(gate, 1u, 2u);
}

__global__ void k_refit_orphans(const uint32_t* parent, uint32_t root, uint32_t end, uint32_t* gate, uint32_t* err) {
    uint32_t i = root + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    if (parent[i] == NONE) bad(gate, err);
}

__device__ __forceinline__ float vload(const uint32_t* p) { return __uint_as_float(*(const volatile uint32_t*)p); }

#ifndef SB_REFIT_ACQREL
#define SB_REFIT_ACQREL 1
#endif
// One node of the node-by-node refit: a leaf's box (and its re-gathered
// triangles), then the climb: the second child to finish computes its parent.
__device__ __forceinline__ void refit_node_climb(uint32_t* nodes, const uint32_t* triIndex, const float* vertexData,
                                                 const uint32_t* triMaterial, const uint32_t* matBits, float4* tris,
                                                 const uint32_t* parent, uint32_t* arrive, uint32_t i, uint4* pairs) {
    uint32_t info = nodes[8 * i + 7];
    if (info == INTERIOR) return;
    uint32_t off = info & 0x00FFFFFFu, cnt = info >> 24;
    if (cnt != 0u) {
        float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
        for (uint32_t t = off; t < off + cnt; ++t) {
            float3 p[3];
            for (int k = 0; k < 3; ++k) {
                const float* v = vertexData + (size_t)triIndex[3 * t + k] * 8u;
                float x = v[0], y = v[1], z = v[2];
                p[k] = make_float3(x, y, z);
                if (x < mnx) mnx = x;
                if (x > mxx) mxx = x;
                if (y < mny) mny = y;
                if (y > mxy) mxy = y;
                if (z < mnz) mnz = z;
                if (z > mxz) mxz = z;
            }
            // re-gather the pre-gathered triangle from the deformed vertices
            tris[3 * t] = make_float4(p[0].x, p[0].y, p[0].z, __uint_as_float(matBits[triMaterial[t]]));
            tris[3 * t + 1] = make_float4(p[1].x, p[1].y, p[1].z, 0.0f);
            tris[3 * t + 2] = make_float4(p[2].x, p[2].y, p[2].z, 0.0f);
        }
        uint32_t* n = nodes + 8 * i;
        n[0] = __float_as_uint(mnx); n[1] = __float_as_uint(mny); n[2] = __float_as_uint(mnz);
        n[3] = __float_as_uint(mxx); n[4] = __float_as_uint(mxy); n[5] = __float_as_uint(mxz);
    }
    uint32_t node = i;
    for (;;) {
        uint32_t p = parent[node];
        if (p == NONE) break;
        // arrival: release publishes this thread's box stores, acquire orders the
        // sibling's box reads below after the sibling's release (one acq_rel atomic)
#if SB_REFIT_ACQREL
        uint32_t prev;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(arrive + p) : "memory");
        if (prev == 0u) break;
#else
        __threadfence();
        if (atomicAdd(&arrive[p], 1u) == 0u) break;
        __threadfence();
#endif
        arrive[p] = 0u;  // both children arrived: ready for the next refit of this range
        uint32_t l = p + 1;
        uint32_t r = *(const volatile uint32_t*)(nodes + 8 * l + 6);
        const uint32_t* L = nodes + 8 * l;
        const uint32_t* R = nodes + 8 * r;
        uint32_t lb[6], rb[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            lb[k] = *(const volatile uint32_t*)(L + k);
            rb[k] = *(const volatile uint32_t*)(R + k);
        }
        uint32_t* n = nodes + 8 * p;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            n[k] = __float_as_uint(js_min(__uint_as_float(lb[k]), __uint_as_float(rb[k])));
            n[3 + k] = __float_as_uint(js_max(__uint_as_float(lb[3 + k]), __uint_as_float(rb[3 + k])));
        }
        if (pairs) store_pair_boxes(pairs + 4u * p, lb, rb);  // the traversal's copy of both child boxes
        node = p;
    }
}

__global__ void k_refit_run(uint32_t* nodes, const uint32_t* triIndex, const float* vertexData,
                            const uint32_t* triMaterial, const uint32_t* matBits, float4* tris,
                            const uint32_t* parent, uint32_t* arrive, uint32_t root, uint32_t end,
                            const uint32_t* gate, uint4* pairs, uint32_t* err) {
    uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    if (*gate == 0u) {
        if (i == root) latch(err, ERR_LAYOUT);  // the range's layout verdict stands until a new upload
        return;
    }
    refit_node_climb(nodes, triIndex, vertexData, triMaterial, matBits, tris, parent, arrive, i, pairs);
}

// Subtrees of at most REFIT_SUB nodes refit inside one CTA: the threaded
// layout stores a node's subtree as [i, miss(i)) (to the range end on the right
// spine), so a CTA takes one such range, computes its leaves, and climbs with
// shared-memory arrival counters; the thread that completes the subtree root
// carries on through the global climb above it. The partition (every node
// whose subtree fits while its parent's does not) is made once per validated
// range, next to the layout checks.
#ifndef SB_REFIT_CTA
#define SB_REFIT_CTA 1
#endif
#ifndef SB_REFIT_SUB
#define SB_REFIT_SUB 256
#endif
constexpr uint32_t REFIT_SUB = SB_REFIT_SUB;  // nodes per CTA subtree (= threads per CTA)

__device__ __forceinline__ uint32_t sub_size(const uint32_t* nodes, uint32_t i, uint32_t end) {
    const uint32_t miss = nodes[8 * i + 6];
    return (miss > i && miss <= end) ? miss - i : end - i;
}

__global__ void k_refit_partition(const uint32_t* nodes, const uint32_t* parent, uint32_t root, uint32_t end,
                                  const uint32_t* gate, uint32_t* subRoots, uint32_t* count) {
    const uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end || *gate != 1u) return;
    if (sub_size(nodes, i, end) > REFIT_SUB) return;
    const uint32_t p = parent[i];
    if (p != NONE && sub_size(nodes, p, end) <= REFIT_SUB) return;
    subRoots[root + atomicAdd(count, 1u)] = i;  // at most end - root entries
}

__global__ void __launch_bounds__(REFIT_SUB) k_refit_cta(uint32_t* nodes, const uint32_t* triIndex,
                                                         const float* vertexData, const uint32_t* triMaterial,
                                                         const uint32_t* matBits, float4* tris,
                                                         const uint32_t* parent, uint32_t* arrive, uint32_t root,
                                                         uint32_t end, const uint32_t* gate, uint4* pairs,
                                                         const uint32_t* subRoots, const uint32_t* count,
                                                         uint32_t* err) {
    __shared__ float sBox[6 * REFIT_SUB];
    __shared__ uint32_t sArr[REFIT_SUB];
    const uint32_t g = *gate;
    if (g == 0u) {
        if (blockIdx.x == 0 && threadIdx.x == 0) latch(err, ERR_LAYOUT);  // the range's verdict stands
        return;
    }
    if (g != 1u) {  // no subtree partition for this layout: node by node, grid-stride
        for (uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x)
            refit_node_climb(nodes, triIndex, vertexData, triMaterial, matBits, tris, parent, arrive, i, pairs);
        return;
    }
    const uint32_t nSub = *count;
    const uint32_t tid = threadIdx.x;
    for (uint32_t t = blockIdx.x; t < nSub; t += gridDim.x) {
        const uint32_t r0 = subRoots[root + t];
        const uint32_t sz = min(sub_size(nodes, r0, end), REFIT_SUB);
        sArr[tid] = 0u;
        __syncthreads();
        uint32_t node = NONE;  // the node this thread carries up
        if (tid < sz) {
            const uint32_t i = r0 + tid;
            const uint32_t info = nodes[8 * i + 7];
            if (info != INTERIOR) {
                const uint32_t off = info & 0x00FFFFFFu, cnt = info >> 24;
                uint32_t* n = nodes + 8 * i;
                if (cnt != 0u) {
                    float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY,
                          mxz = -INFINITY;
                    for (uint32_t tr = off; tr < off + cnt; ++tr) {
                        float3 p[3];
                        for (int k = 0; k < 3; ++k) {
                            const float* v = vertexData + (size_t)triIndex[3 * tr + k] * 8u;
                            const float x = v[0], y = v[1], z = v[2];
                            p[k] = make_float3(x, y, z);
                            if (x < mnx) mnx = x;
                            if (x > mxx) mxx = x;
                            if (y < mny) mny = y;
                            if (y > mxy) mxy = y;
                            if (z < mnz) mnz = z;
                            if (z > mxz) mxz = z;
                        }
                        tris[3 * tr] = make_float4(p[0].x, p[0].y, p[0].z, __uint_as_float(matBits[triMaterial[tr]]));
                        tris[3 * tr + 1] = make_float4(p[1].x, p[1].y, p[1].z, 0.0f);
                        tris[3 * tr + 2] = make_float4(p[2].x, p[2].y, p[2].z, 0.0f);
                    }
                    n[0] = __float_as_uint(mnx); n[1] = __float_as_uint(mny); n[2] = __float_as_uint(mnz);
                    n[3] = __float_as_uint(mxx); n[4] = __float_as_uint(mxy); n[5] = __float_as_uint(mxz);
                }
                for (int k = 0; k < 6; ++k) sBox[6 * tid + k] = __uint_as_float(n[k]);
                node = i;
            }
        }
        // inside the subtree: the second child to finish computes its parent
        volatile float* vb = sBox;
        while (node != NONE && node != r0) {
            const uint32_t p = parent[node];
            const uint32_t pl = p - r0;  // p lies in [r0, node): the subtree is [r0, r0 + sz)
            if (p == NONE || pl >= sz) {  // a partition that does not match the layout
                latch(err, ERR_LAYOUT);
                node = NONE;
                break;
            }
            __threadfence_block();
            if (atomicAdd(&sArr[pl], 1u) == 0u) {
                node = NONE;
                break;
            }
            __threadfence_block();
            const uint32_t l = p + 1, r = nodes[8 * l + 6];
            const uint32_t ll = l - r0, rl = r - r0;
            if (ll >= sz || rl >= sz) {
                latch(err, ERR_LAYOUT);
                node = NONE;
                break;
            }
            uint32_t lb[6], rb[6];
            for (int k = 0; k < 6; ++k) {
                lb[k] = __float_as_uint(vb[6 * ll + k]);
                rb[k] = __float_as_uint(vb[6 * rl + k]);
            }
            uint32_t* n = nodes + 8 * p;
            for (int k = 0; k < 3; ++k) {
                const float mn = js_min(__uint_as_float(lb[k]), __uint_as_float(rb[k]));
                const float mx = js_max(__uint_as_float(lb[3 + k]), __uint_as_float(rb[3 + k]));
                n[k] = __float_as_uint(mn);
                n[3 + k] = __float_as_uint(mx);
                vb[6 * pl + k] = mn;
                vb[6 * pl + 3 + k] = mx;
            }
            if (pairs) store_pair_boxes(pairs + 4u * p, lb, rb);
            node = p;
        }
        // the subtree root is done: the levels above through global memory
        while (node != NONE) {
            const uint32_t p = parent[node];
            if (p == NONE) break;
            uint32_t prev;
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(arrive + p) : "memory");
            if (prev == 0u) break;
            arrive[p] = 0u;
            const uint32_t l = p + 1;
            const uint32_t r = *(const volatile uint32_t*)(nodes + 8 * l + 6);
            const uint32_t* L = nodes + 8 * l;
            const uint32_t* Rn = nodes + 8 * r;
            uint32_t lb[6], rb[6];
            for (int k = 0; k < 6; ++k) {
                lb[k] = *(const volatile uint32_t*)(L + k);
                rb[k] = *(const volatile uint32_t*)(Rn + k);
            }
            uint32_t* n = nodes + 8 * p;
            for (int k = 0; k < 3; ++k) {
                n[k] = __float_as_uint(js_min(__uint_as_float(lb[k]), __uint_as_float(rb[k])));
                n[3 + k] = __float_as_uint(js_max(__uint_as_float(lb[3 + k]), __uint_as_float(rb[3 + k])));
            }
            if (pairs) store_pair_boxes(pairs + 4u * p, lb, rb);
            node = p;
        }
        __syncthreads();  // the shared arrays serve the next subtree
    }
}

__global__ void k_scatter_vertices(float* v8, const float* p3, const float* n3, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* v = v8 + 8u * (size_t)i;
    v[0] = p3[3u * (size_t)i];
    v[1] = p3[3u * (size_t)i + 1u];
    v[2] = p3[3u * (size_t)i + 2u];
    if (n3) {
        v[3] = n3[3u * (size_t)i];
        v[4] = n3[3u * (size_t)i + 1u];
        v[5] = n3[3u * (size_t)i + 2u];
    }
}

cudaError_t launch_scatter_vertices(float* vertexData8, const float* positions, const float* normals, uint32_t n,
                                    cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_scatter_vertices<<<(n + 255) / 256, 256, 0, st>>>(vertexData8, positions, normals, n);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_refit_blas(const SceneBuffers& B, uint32_t root, uint32_t end, uint32_t* err, uint32_t* gate,
                              cudaStream_t st, bool validated) {
    if (end <= root) return cudaSuccess;
    uint32_t n = end - root;
    unsigned g = (n + 255) / 256;
    if (!validated) {
        cudaError_t e = cudaMemsetAsync(gate, 1, sizeof(uint32_t), st);  // nonzero: valid until a check fails
        if (e != cudaSuccess) return e;
        k_refit_reset<<<g, 256, 0, st>>>(B.parent, B.arrive, root, end); note_launch();
        k_refit_link<<<g, 256, 0, st>>>(B.nodes, B.triIndex, B.triMaterial, B.triCount, B.vertexCount,
                                        B.materialCount, B.parent, root, end, gate, err); note_launch();
        k_refit_orphans<<<g, 256, 0, st>>>(B.parent, root, end, gate, err); note_launch();
        if (SB_REFIT_CTA) {
            cudaError_t e2 = cudaMemsetAsync(gate + 16, 0, sizeof(uint32_t), st);  // the range's subtree count
            if (e2 != cudaSuccess) return e2;
            k_refit_partition<<<g, 256, 0, st>>>(B.nodes, B.parent, root, end, gate, B.subRoots, gate + 16);
            note_launch();
        }
    }
    if (SB_REFIT_CTA) {
        // one CTA per subtree (the count is on the device; idle CTAs return at once)
        const unsigned ctas = n < 1184u ? n : 1184u;
        k_refit_cta<<<ctas, REFIT_SUB, 0, st>>>(B.nodes, B.triIndex, B.vertexData, B.triMaterial, B.matBits, B.tris,
                                                B.parent, B.arrive, root, end, gate, B.pairs, B.subRoots, gate + 16,
                                                err);
        note_launch();
        return cudaGetLastError();
    }
    k_refit_run<<<g, 256, 0, st>>>(B.nodes, B.triIndex, B.vertexData, B.triMaterial, B.matBits, B.tris, B.parent,
                                   B.arrive, root, end, gate, B.pairs, err); note_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------- instance math (FP64)
// Operation order is fixed and every product/sum separately rounded, so the
// results are reproducible bit-for-bit by a host evaluation in the same order.
#define DM(a, b) __dmul_rn((a), (b))
#define DA(a, b) __dadd_rn((a), (b))
#define DS(a, b) __dsub_rn((a), (b))

__device__ __forceinline__ double mat(const double* m, int r, int c) { return m[c * 4 + r]; }

__device__ double det4(const double* m) {
    double s01 = DS(DM(mat(m, 2, 0), mat(m, 3, 1)), DM(mat(m, 2, 1), mat(m, 3, 0)));
    double s02 = DS(DM(mat(m, 2, 0), mat(m, 3, 2)), DM(mat(m, 2, 2), mat(m, 3, 0)));
    double s03 = DS(DM(mat(m, 2, 0), mat(m, 3, 3)), DM(mat(m, 2, 3), mat(m, 3, 0)));
    double s12 = DS(DM(mat(m, 2, 1), mat(m, 3, 2)), DM(mat(m, 2, 2), mat(m, 3, 1)));
    double s13 = DS(DM(mat(m, 2, 1), mat(m, 3, 3)), DM(mat(m, 2, 3), mat(m, 3, 1)));
    double s23 = DS(DM(mat(m, 2, 2), mat(m, 3, 3)), DM(mat(m, 2, 3), mat(m, 3, 2)));
    double c0 = DA(DS(DM(mat(m, 1, 1), s23), DM(mat(m, 1, 2), s13)), DM(mat(m, 1, 3), s12));
    double c1 = DA(DS(DM(mat(m, 1, 0), s23), DM(mat(m, 1, 2), s03)), DM(mat(m, 1, 3), s02));
    double c2 = DA(DS(DM(mat(m, 1, 0), s13), DM(mat(m, 1, 1), s03)), DM(mat(m, 1, 3), s01));
    double c3 = DA(DS(DM(mat(m, 1, 0), s12), DM(mat(m, 1, 1), s02)), DM(mat(m, 1, 2), s01));
    return DS(DA(DS(DM(mat(m, 0, 0), c0), DM(mat(m, 0, 1), c1)), DM(mat(m, 0, 2), c2)), DM(mat(m, 0, 3), c3));
}

// First three rows of the inverse (adjugate / determinant), zeros if singular.
__device__ void inverse_rows(const double* m, double out[12]) {
    double det = det4(m);
    if (det == 0.0) {
        for (int i = 0; i < 12; ++i) out[i] = 0.0;
        return;
    }
    double inv = __ddiv_rn(1.0, det);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) {
            int rows[3], cols[3];
            for (int i = 0, k = 0; i < 4; ++i) if (i != c) rows[k++] = i;
            for (int j = 0, k = 0; j < 4; ++j) if (j != r) cols[k++] = j;
            double t0 = DM(mat(m, rows[0], cols[0]),
                           DS(DM(mat(m, rows[1], cols[1]), mat(m, rows[2], cols[2])),
                              DM(mat(m, rows[1], cols[2]), mat(m, rows[2], cols[1]))));
            double t1 = DM(mat(m, rows[0], cols[1]),
                           DS(DM(mat(m, rows[1], cols[0]), mat(m, rows[2], cols[2])),
                              DM(mat(m, rows[1], cols[2]), mat(m, rows[2], cols[0]))));
            double t2 = DM(mat(m, rows[0], cols[2]),
                           DS(DM(mat(m, rows[1], cols[0]), mat(m, rows[2], cols[1])),
                              DM(mat(m, rows[1], cols[1]), mat(m, rows[2], cols[0]))));
            double m3 = DA(DS(t0, t1), t2);
            double cof = ((r + c) & 1) ? -m3 : m3;
            out[r * 4 + c] = DM(cof, inv);
        }
}

__device__ void transform_box(const double* m, const double lmin[3], const double lmax[3], double wmin[3],
                              double wmax[3]) {
    for (int a = 0; a < 3; ++a) { wmin[a] = INFINITY; wmax[a] = -INFINITY; }
    for (int i = 0; i < 8; ++i) {
        double x = (i & 1) ? lmax[0] : lmin[0];
        double y = (i & 2) ? lmax[1] : lmin[1];
        double z = (i & 4) ? lmax[2] : lmin[2];
        double w = __ddiv_rn(1.0, DA(DA(DA(DM(m[3], x), DM(m[7], y)), DM(m[11], z)), m[15]));
        double p[3] = {DM(DA(DA(DA(DM(m[0], x), DM(m[4], y)), DM(m[8], z)), m[12]), w),
                       DM(DA(DA(DA(DM(m[1], x), DM(m[5], y)), DM(m[9], z)), m[13]), w),
                       DM(DA(DA(DA(DM(m[2], x), DM(m[6], y)), DM(m[10], z)), m[14]), w)};
        for (int a = 0; a < 3; ++a) {
            if (p[a] < wmin[a]) wmin[a] = p[a];
            if (p[a] > wmax[a]) wmax[a] = p[a];
        }
    }
}

// computeDynamic for one source instance: inverse rows, winding sign, FP64 AABB.
__device__ void compute_instance(const SceneBuffers& B, const InstanceTable& I, uint32_t src, uint32_t* err) {
    const double* m = I.world + (size_t)src * 16u;
    double inv[12];
    inverse_rows(m, inv);
    for (int k = 0; k < 12; ++k) I.invRows[(size_t)src * 12u + k] = __double2float_rn(inv[k]);
    I.detSign[src] = det4(m) < 0.0 ? -1.0f : 1.0f;
    double mn[3], mx[3];
    uint32_t root = I.blasRoot[src], end = I.blasEnd[src];
    if (I.active[src]) {
        if (!(root < end && end <= B.nodeCount)) {
            latch(err, ERR_LAYOUT);
            for (int a = 0; a < 3; ++a) mn[a] = mx[a] = 0.0;
        } else {
            const float* nb = reinterpret_cast<const float*>(B.nodes + (size_t)root * 8u);
            double lmin[3] = {nb[0], nb[1], nb[2]}, lmax[3] = {nb[3], nb[4], nb[5]};
            transform_box(m, lmin, lmax, mn, mx);
        }
    } else {
        for (int a = 0; a < 3; ++a) mn[a] = mx[a] = m[12 + a];
    }
    double* o = I.aabb + (size_t)src * 9u;
    for (int a = 0; a < 3; ++a) {
        o[a] = mn[a];
        o[3 + a] = mx[a];
        o[6 + a] = DM(DA(mn[a], mx[a]), 0.5);
        if (o[6 + a] != o[6 + a]) latch(err, ERR_NAN_KEY);
    }
}

// writeDynamic's instance record for one slot (spectral_scene.js:1340-1355),
// into both the reference tail and the derived instance rows.
__device__ void write_slot(const SceneBuffers& B, const InstanceTable& I, uint32_t slot, uint32_t src, bool rows) {
    const double* a = I.aabb + (size_t)src * 9u;
    float* lb = I.liveBounds + (size_t)slot * 6u;
    for (int k = 0; k < 6; ++k) lb[k] = __double2float_rn(a[k]);
    if (!rows) return;
    float* R = B.materials + B.instBase + (size_t)slot * 28u;
    const float* ir = I.invRows + (size_t)src * 12u;
    for (int k = 0; k < 12; ++k) R[k] = ir[k];
    R[12] = float(I.blasRoot[src]);
    R[13] = float(I.blasEnd[src]);
    R[14] = I.detSign[src];
    R[15] = I.active[src] ? 1.0f : 0.0f;
    for (int k = 16; k < 28; ++k) R[k] = 0.0f;
    B.inst[4 * slot] = make_float4(ir[0], ir[1], ir[2], ir[3]);
    B.inst[4 * slot + 1] = make_float4(ir[4], ir[5], ir[6], ir[7]);
    B.inst[4 * slot + 2] = make_float4(ir[8], ir[9], ir[10], ir[11]);
    B.inst[4 * slot + 3] = make_float4(__uint_as_float(I.blasRoot[src]), __uint_as_float(I.blasEnd[src]),
                                       I.detSign[src], I.active[src] ? 1.0f : 0.0f);
}

__device__ __forceinline__ void write_tlas_node(const SceneBuffers& B, uint32_t idx, const float bx[6], uint32_t miss,
                                                uint32_t off, uint32_t cnt) {
    float* N = B.materials + B.tlasBase + (size_t)idx * 12u;
    for (int k = 0; k < 6; ++k) N[k] = bx[k];
    N[6] = float(miss);
    N[7] = cnt ? float(off) : 0.0f;
    N[8] = float(cnt);
    N[9] = N[10] = N[11] = 0.0f;
    B.tlas[2 * idx] = make_uint4(__float_as_uint(bx[0]), __float_as_uint(bx[1]), __float_as_uint(bx[2]),
                                 __float_as_uint(bx[3]));
    B.tlas[2 * idx + 1] = make_uint4(__float_as_uint(bx[4]), __float_as_uint(bx[5]), miss, (cnt << 24) | (cnt ? off : 0u));
}

// ------------------------------------------------------------- TLAS build
// Order-preserving 64-bit key of a double (-0 folded onto +0, as the reference
// comparator c[a] - c[b] treats them as equal).
__device__ __forceinline__ unsigned long long sortable(double d) {
    if (d == 0.0) d = 0.0;
    unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// Sort record: (group << 13 | position) and key; ordered by group, then key,
// then position, so ties keep the current order (a stable sort) and groups
// stay in place.
struct BuildRec {
    unsigned long long key;
    uint32_t segpos;
    uint32_t pad;
};
__device__ __forceinline__ bool rec_less(const BuildRec& a, const BuildRec& b) {
    uint32_t sa = a.segpos >> 13, sb = b.segpos >> 13;
    if (sa != sb) return sa < sb;
    if (a.key != b.key) return a.key < b.key;
    return (a.segpos & 0x1FFFu) < (b.segpos & 0x1FFFu);
}

// min with ties kept by the earlier position; NaN never selected (the strict
// `<` scan of buildTlasRecords from +Infinity)
__device__ __forceinline__ void red_min(double& v, uint32_t& p, double v2, uint32_t p2) {
    if (v2 != v2) return;
    if (v != v || v2 < v || (v2 == v && p2 < p)) { v = v2; p = p2; }
}
__device__ __forceinline__ void red_max(double& v, uint32_t& p, double v2, uint32_t p2) {
    if (v2 != v2) return;
    if (v != v || v2 > v || (v2 == v && p2 < p)) { v = v2; p = p2; }
}

struct Seg { uint16_t lo, hi, idx; };

// Up to this many instances a level orders its segments by rank (the summed
// squared segment lengths stay below n^2 / 2 per level); above it by one
// bitonic sort of all positions per level.
constexpr uint32_t TLAS_RANK_SORT_MAX = 512;

__host__ __device__ inline size_t tlas_build_smem(uint32_t n) {
    uint32_t P = 1;
    while (P < n) P <<= 1;
    size_t b = (size_t)P * sizeof(BuildRec) + (size_t)n * 4u * 3u + 4u + (size_t)n * sizeof(Seg) * 2u;
    return (b + 15u) & ~(size_t)15u;
}

__global__ void __launch_bounds__(1024) k_tlas_build(SceneBuffers B, InstanceTable I, uint32_t* err) {
    extern __shared__ unsigned char smem[];
    const uint32_t n = I.count;
    uint32_t P = 1;
    while (P < n) P <<= 1;
    BuildRec* rec = reinterpret_cast<BuildRec*>(smem);                       // P
    uint32_t* order = reinterpret_cast<uint32_t*>(rec + P);                  // n
    uint32_t* segOf = order + n;                                             // n (also a gather buffer)
    uint32_t* nodesTab = segOf + n;                                          // n+1
    Seg* segA = reinterpret_cast<Seg*>(nodesTab + n + 1);                    // n
    Seg* segB = segA + n;                                                    // n
    __shared__ uint32_t nSeg, nNext, level;
    __shared__ uint8_t axisOf[TLAS_BUILD_MAX];

    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        compute_instance(B, I, i, err);
        order[i] = i;
    }
    if (threadIdx.x == 0) {
        // subtree node counts of the median split with leaf size 2
        nodesTab[0] = 1;
        for (uint32_t m = 1; m <= n; ++m) nodesTab[m] = m <= 2 ? 1u : 1u + nodesTab[m >> 1] + nodesTab[m - (m >> 1)];
        segA[0] = Seg{0, (uint16_t)n, 0};
        nSeg = 1;
        level = 0;
    }
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nWarps = blockDim.x >> 5;
    Seg* cur = segA;
    Seg* nxt = segB;
    while (nSeg > 0) {
        // positions whose leaf was emitted at an earlier level belong to no segment
        for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) segOf[j] = NONE;
        __syncthreads();
        // (a) bounds + node record per segment, one warp per segment
        for (uint32_t s = warp; s < nSeg; s += nWarps) {
            Seg sg = cur[s];
            double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t pmn[3] = {NONE, NONE, NONE}, pmx[3] = {NONE, NONE, NONE};
            for (uint32_t j = sg.lo + lane; j < sg.hi; j += 32) {
                const double* a = I.aabb + (size_t)order[j] * 9u;
                for (int k = 0; k < 3; ++k) {
                    red_min(mn[k], pmn[k], a[k], j);
                    red_max(mx[k], pmx[k], a[3 + k], j);
                }
                segOf[j] = s;
            }
            for (int off = 16; off > 0; off >>= 1)
                for (int k = 0; k < 3; ++k) {
                    double v = __shfl_down_sync(0xFFFFFFFFu, mn[k], off);
                    uint32_t p = __shfl_down_sync(0xFFFFFFFFu, pmn[k], off);
                    if (p != NONE) red_min(mn[k], pmn[k], v, p);
                    v = __shfl_down_sync(0xFFFFFFFFu, mx[k], off);
                    p = __shfl_down_sync(0xFFFFFFFFu, pmx[k], off);
                    if (p != NONE) red_max(mx[k], pmx[k], v, p);
                }
            if (lane == 0) {
                float bx[6];
                for (int k = 0; k < 3; ++k) {
                    bx[k] = __double2float_rn(mn[k]);
                    bx[3 + k] = __double2float_rn(mx[k]);
                }
                uint32_t cnt = (uint32_t)sg.hi - sg.lo;
                uint32_t miss = sg.idx + nodesTab[cnt];
                if (cnt <= 2) {
                    write_tlas_node(B, sg.idx, bx, miss, sg.lo, cnt);
                    axisOf[s] = 255;
                } else {
                    write_tlas_node(B, sg.idx, bx, miss, 0, 0);
                    double ex = DS(mx[0], mn[0]), ey = DS(mx[1], mn[1]), ez = DS(mx[2], mn[2]);
                    axisOf[s] = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
                }
                I.nodeDepth[sg.idx] = level;
            }
        }
        __syncthreads();
        if (n <= TLAS_RANK_SORT_MAX) {
            // (b) the stable order of every interior segment by its split axis's FP64
            // centroid key: each position's rank among its segment's positions by
            // (key, position), one thread per position; leaf segments and finished
            // positions keep their place. The keys are staged once per level.
            unsigned long long* keys = reinterpret_cast<unsigned long long*>(rec);  // n keys, then n slots
            uint32_t* newOrder = reinterpret_cast<uint32_t*>(keys + n);
            for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
                const uint32_t s = segOf[j];
                const uint32_t ax = s == NONE ? 255u : axisOf[s];
                keys[j] = ax == 255u ? 0ull : sortable(I.aabb[(size_t)order[j] * 9u + 6u + ax]);
            }
            __syncthreads();
            for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
                const uint32_t s = segOf[j];
                uint32_t dest = j;
                if (s != NONE && axisOf[s] != 255u) {
                    const uint32_t lo = cur[s].lo, hi = cur[s].hi;
                    const unsigned long long kj = keys[j];
                    uint32_t r = 0;
                    for (uint32_t q = lo; q < hi; ++q) {
                        const unsigned long long kq = keys[q];
                        r += (kq < kj || (kq == kj && q < j)) ? 1u : 0u;
                    }
                    dest = lo + r;
                }
                newOrder[dest] = order[j];
            }
            __syncthreads();
            for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) order[j] = newOrder[j];
        } else {
            // (b) sort records grouped by the first position of their segment (or by their
            // own position when finished), so every group stays inside its range; leaf
            // segments and finished positions keep their order (constant key)
            for (uint32_t j = threadIdx.x; j < P; j += blockDim.x) {
                BuildRec r;
                if (j < n) {
                    uint32_t s = segOf[j];
                    uint32_t ax = s == NONE ? 255u : axisOf[s];
                    uint32_t group = s == NONE ? j : (uint32_t)cur[s].lo;
                    r.segpos = (group << 13) | j;
                    r.key = ax == 255 ? 0ull : sortable(I.aabb[(size_t)order[j] * 9u + 6u + ax]);
                } else {
                    r.segpos = 0xFFFFFFFFu;
                    r.key = ~0ull;
                }
                r.pad = 0;
                rec[j] = r;
            }
            __syncthreads();
            // (c) bitonic sort of P records
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
                    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                        uint32_t ixj = i ^ jj;
                        if (ixj > i) {
                            bool up = (i & k) == 0;
                            BuildRec a = rec[i], b = rec[ixj];
                            bool sw = up ? rec_less(b, a) : rec_less(a, b);
                            if (sw) { rec[i] = b; rec[ixj] = a; }
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) segOf[j] = order[rec[j].segpos & 0x1FFFu];
            __syncthreads();
            for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) order[j] = segOf[j];
        }
        // (d) children of interior segments, in order of lo
        if (threadIdx.x == 0) {
            uint32_t m = 0;
            for (uint32_t s = 0; s < nSeg; ++s) {
                Seg sg = cur[s];
                if ((uint32_t)sg.hi - sg.lo <= 2) continue;
                uint32_t mid = ((uint32_t)sg.lo + sg.hi) >> 1;
                nxt[m++] = Seg{sg.lo, (uint16_t)mid, (uint16_t)(sg.idx + 1)};
                nxt[m++] = Seg{(uint16_t)mid, sg.hi, (uint16_t)(sg.idx + 1 + nodesTab[mid - sg.lo])};
            }
            nNext = m;
            level = level + 1;
        }
        __syncthreads();
        Seg* t = cur; cur = nxt; nxt = t;
        if (threadIdx.x == 0) nSeg = nNext;
        __syncthreads();
    }
    if (threadIdx.x == 0) *I.scratch = level - 1;
    // (e) slots: order, inverse map, instance records, live bounds
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        uint32_t src = order[s];
        I.order[s] = src;
        I.slotOf[src] = s;
        write_slot(B, I, s, src, true);
    }
}

cudaError_t launch_tlas_build(const SceneBuffers& B, const InstanceTable& I, uint32_t* err, cudaStream_t st) {
    uint32_t n = I.count;
    if (n == 0 || n > TLAS_BUILD_MAX) return cudaErrorInvalidValue;
    size_t smem = tlas_build_smem(n);
    cudaError_t e = cudaFuncSetAttribute(k_tlas_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_tlas_build<<<1, 1024, smem, st>>>(B, I, err); note_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------ transform lane
// updateTransforms (spectral_scene.js:1402-1514): recompute the listed source
// instances (all when srcList is null) and write their slots.
__global__ void k_update_instances(SceneBuffers B, InstanceTable I, const uint32_t* srcList, const double* world16,
                                   uint32_t count, int rewriteRows, uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t total = srcList ? count : I.count;
    if (i >= total) return;
    uint32_t src = srcList ? srcList[i] : i;
    if (src >= I.count) { latch(err, ERR_LAYOUT); return; }
    if (srcList && world16)
        for (int k = 0; k < 16; ++k) I.world[(size_t)src * 16u + k] = world16[(size_t)i * 16u + k];
    compute_instance(B, I, src, err);
    write_slot(B, I, I.slotOf[src], src, rewriteRows != 0);
}

cudaError_t launch_update_instances(const SceneBuffers& B, const InstanceTable& I, const uint32_t* srcList,
                                    const double* world16, uint32_t count, int rewriteRows, uint32_t* err,
                                    cudaStream_t st) {
    uint32_t total = srcList ? count : I.count;
    if (total == 0) return cudaSuccess;
    k_update_instances<<<(total + 127) / 128, 128, 0, st>>>(B, I, srcList, world16, count, rewriteRows, err); note_launch();
    return cudaGetLastError();
}

// refitFlatTlasRange over the frozen partition, deepest level first (the
// body of one CTA; the caller's writes to liveBounds precede a barrier).
// The level pass on the records in global memory (larger TLASes).
__device__ __forceinline__ void tlas_refit_levels(const SceneBuffers& B, const InstanceTable& I, uint32_t nn,
                                                  int maxDepth) {
    for (int d = maxDepth; d >= 0; --d) {
        for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) {
            if (I.nodeDepth[i] != (uint32_t)d) continue;
            float* N = B.materials + B.tlasBase + (size_t)i * 12u;
            float bx[6];
            uint32_t miss = (uint32_t)N[6];
            float cf = N[8];
            if (cf > 0.0f) {
                uint32_t off = (uint32_t)N[7], cnt = (uint32_t)cf;
                float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
                for (uint32_t s = off; s < off + cnt; ++s) {
                    const float* b = I.liveBounds + (size_t)s * 6u;
                    for (int k = 0; k < 3; ++k) {
                        if (b[k] < mn[k]) mn[k] = b[k];
                        if (b[3 + k] > mx[k]) mx[k] = b[3 + k];
                    }
                }
                for (int k = 0; k < 3; ++k) { bx[k] = mn[k]; bx[3 + k] = mx[k]; }
                write_tlas_node(B, i, bx, miss, off, cnt);
            } else {
                const float* L = B.materials + B.tlasBase + (size_t)(i + 1) * 12u;
                const float* R = B.materials + B.tlasBase + (size_t)((uint32_t)L[6]) * 12u;
                for (int k = 0; k < 3; ++k) {
                    bx[k] = js_min(L[k], R[k]);
                    bx[3 + k] = js_max(L[3 + k], R[3 + k]);
                }
                write_tlas_node(B, i, bx, miss, 0, 0);
            }
        }
        __syncthreads();
    }
}

// The traversal's child-pair copy of the refit bounds (entries are structural).
__device__ __forceinline__ void tlas_refit_pairs(const SceneBuffers& B, uint32_t nn) {
    if (!B.tlasPairs) return;
    for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) {
        uint4 b = B.tlas[2 * i + 1];
        if ((b.w >> 24) != 0u || i + 1 >= nn) continue;
        uint32_t l = i + 1, r = B.tlas[2 * l + 1].z;
        if (!(r > l && r < nn)) continue;
        uint4 la = B.tlas[2 * l], lb = B.tlas[2 * l + 1], ra = B.tlas[2 * r], rb = B.tlas[2 * r + 1];
        const uint32_t b0[6] = {la.x, la.y, la.z, la.w, lb.x, lb.y};
        const uint32_t b1[6] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y};
        store_pair_boxes(B.tlasPairs + 4u * i, b0, b1);
    }
}

// TLASes of up to this many nodes run the level pass on a shared-memory copy
// of the boxes, structure words and depths (the same min / max on the same
// values; every node is still written to the records as it is refit), so a
// level reads its children from shared memory instead of global memory.
#ifndef SB_TLAS_STAGE_NODES
#define SB_TLAS_STAGE_NODES 512
#endif
constexpr uint32_t TLAS_STAGE_NODES = SB_TLAS_STAGE_NODES > 0 ? SB_TLAS_STAGE_NODES : 1;

__device__ __forceinline__ void tlas_refit_body(const SceneBuffers& B, const InstanceTable& I) {
    const uint32_t nn = B.tlasNodeCount;
    const int maxDepth = (int)*(volatile uint32_t*)I.scratch;
    if (SB_TLAS_STAGE_NODES > 0 && nn <= TLAS_STAGE_NODES) {
        __shared__ float sBox[6 * TLAS_STAGE_NODES];
        __shared__ uint32_t sMiss[TLAS_STAGE_NODES], sOff[TLAS_STAGE_NODES], sCnt[TLAS_STAGE_NODES],
            sDepth[TLAS_STAGE_NODES];
        const float* T = B.materials + B.tlasBase;
        for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) {
            const float* N = T + (size_t)i * 12u;
            for (int k = 0; k < 6; ++k) sBox[6 * i + k] = N[k];
            sMiss[i] = (uint32_t)N[6];
            sOff[i] = (uint32_t)N[7];
            sCnt[i] = N[8] > 0.0f ? (uint32_t)N[8] : 0u;
            sDepth[i] = I.nodeDepth[i];
        }
        __syncthreads();
        for (int d = maxDepth; d >= 0; --d) {
            for (uint32_t i = threadIdx.x; i < nn; i += blockDim.x) {
                if (sDepth[i] != (uint32_t)d) continue;
                float bx[6];
                const uint32_t cnt = sCnt[i];
                if (cnt > 0u) {
                    const uint32_t off = sOff[i];
                    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
                    for (uint32_t s = off; s < off + cnt; ++s) {
                        const float* b = I.liveBounds + (size_t)s * 6u;
                        for (int k = 0; k < 3; ++k) {
                            if (b[k] < mn[k]) mn[k] = b[k];
                            if (b[3 + k] > mx[k]) mx[k] = b[3 + k];
                        }
                    }
                    for (int k = 0; k < 3; ++k) { bx[k] = mn[k]; bx[3 + k] = mx[k]; }
                } else {
                    const uint32_t l = i + 1, r = sMiss[l];
                    for (int k = 0; k < 3; ++k) {
                        bx[k] = js_min(sBox[6 * l + k], sBox[6 * r + k]);
                        bx[3 + k] = js_max(sBox[6 * l + 3 + k], sBox[6 * r + 3 + k]);
                    }
                }
                for (int k = 0; k < 6; ++k) sBox[6 * i + k] = bx[k];
                write_tlas_node(B, i, bx, sMiss[i], sOff[i], cnt);
            }
            __syncthreads();
        }
    } else {
        tlas_refit_levels(B, I, nn, maxDepth);
    }
    tlas_refit_pairs(B, nn);
}

__global__ void __launch_bounds__(1024) k_tlas_refit(SceneBuffers B, InstanceTable I) { tlas_refit_body(B, I); }

// The transform lane in one CTA: the listed (or every) source instance's rows
// and bounds, then the TLAS refit over them, with one launch.
__global__ void __launch_bounds__(512) k_update_refit_tlas(SceneBuffers B, InstanceTable I, const uint32_t* srcList,
                                                            const double* world16, uint32_t count, int rewriteRows,
                                                            uint32_t* err) {
    const uint32_t total = srcList ? count : I.count;
    for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
        const uint32_t src = srcList ? srcList[i] : i;
        if (src >= I.count) {
            latch(err, ERR_LAYOUT);
            continue;
        }
        if (srcList && world16)
            for (int k = 0; k < 16; ++k) I.world[(size_t)src * 16u + k] = world16[(size_t)i * 16u + k];
        compute_instance(B, I, src, err);
        write_slot(B, I, I.slotOf[src], src, rewriteRows != 0);
    }
    __syncthreads();
    tlas_refit_body(B, I);
}

// Depth of every TLAS node and the refit-index checks of
// createFlatTlasRefitIndex (gi_refit.js:298-346); one thread, structural
// changes only.
__global__ void k_tlas_index(SceneBuffers B, InstanceTable I, uint32_t* owner, uint32_t* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t nn = B.tlasNodeCount, ic = B.instCount;
    for (uint32_t i = 0; i < nn; ++i) I.nodeDepth[i] = NONE;
    for (uint32_t s = 0; s < ic; ++s) owner[s] = NONE;
    uint32_t maxD = 0;
    if (nn) I.nodeDepth[0] = 0;
    for (uint32_t i = 0; i < nn; ++i) {
        const float* N = B.materials + B.tlasBase + (size_t)i * 12u;
        uint32_t d = I.nodeDepth[i];
        if (d == NONE) { latch(err, ERR_LAYOUT); return; }
        if (d > maxD) maxD = d;
        float cf = N[8];
        if (cf > 0.0f) {
            float off = N[7];
            if (!(off >= 0.0f) || floorf(off) != off || floorf(cf) != cf || off + cf > (float)ic) {
                latch(err, ERR_LAYOUT);
                return;
            }
            for (uint32_t s = (uint32_t)off; s < (uint32_t)(off + cf); ++s) {
                if (owner[s] != NONE) { latch(err, ERR_LAYOUT); return; }
                owner[s] = i;
            }
        } else {
            uint32_t l = i + 1;
            if (l >= nn) { latch(err, ERR_LAYOUT); return; }
            float rf = B.materials[B.tlasBase + (size_t)l * 12u + 6u];
            if (floorf(rf) != rf || !(rf > (float)l && rf < (float)nn)) { latch(err, ERR_LAYOUT); return; }
            uint32_t r = (uint32_t)rf;
            if (I.nodeDepth[l] != NONE || I.nodeDepth[r] != NONE) { latch(err, ERR_LAYOUT); return; }
            I.nodeDepth[l] = d + 1;
            I.nodeDepth[r] = d + 1;
        }
    }
    for (uint32_t s = 0; s < ic; ++s)
        if (owner[s] == NONE) { latch(err, ERR_LAYOUT); return; }
    *I.scratch = maxD;
}

cudaError_t launch_update_refit_tlas(const SceneBuffers& B, const InstanceTable& I, const uint32_t* srcList,
                                     const double* world16, uint32_t count, int rewriteRows, uint32_t* err,
                                     cudaStream_t st) {
    k_update_refit_tlas<<<1, 512, 0, st>>>(B, I, srcList, world16, count, rewriteRows, err); note_launch();
    return cudaGetLastError();
}

cudaError_t launch_tlas_refit(const SceneBuffers& B, const InstanceTable& I, uint32_t* err, cudaStream_t st) {
    if (B.tlasNodeCount == 0) return cudaSuccess;
    k_tlas_refit<<<1, 1024, 0, st>>>(B, I); note_launch();
    return cudaGetLastError();
}

cudaError_t launch_tlas_index(const SceneBuffers& B, const InstanceTable& I, uint32_t* owner, uint32_t* err,
                              cudaStream_t st) {
    k_tlas_index<<<1, 32, 0, st>>>(B, I, owner, err); note_launch();
    return cudaGetLastError();
}

}  // namespace sb
