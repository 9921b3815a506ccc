// sb_pairs.cu — structural derivation of the child-pair nodes that the
// traversal walks (layout in sb_internal.cuh) and of the deepest node of the
// BLASes and of the TLAS, which bounds the traversal stack.
//
// The reference nodes stay the wire format: a pair node copies the bounds of
// an interior node's two children (left = index + 1, right = the left child's
// miss link, the threaded layout of spectral_traverse.js:354-435) bit for bit,
// so a box test on a pair gives exactly the reference's box test on the child.
#include "sb_pairs.cuh"
#include "sb_kernels.cuh"

namespace sb {

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t DEPTH_LIMIT = 64u;  // deeper trees use the stackless walk

__device__ __forceinline__ void node_box(const uint32_t* nodes, uint32_t i, uint32_t b[6]) {
    const uint4* p = reinterpret_cast<const uint4*>(nodes + 8u * i);
    uint4 a = p[0], c = p[1];
    b[0] = a.x; b[1] = a.y; b[2] = a.z; b[3] = a.w; b[4] = c.x; b[5] = c.y;
}

__global__ void k_blas_link_all(const uint32_t* nodes, uint32_t n, uint32_t* parent) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[8u * i + 7u] != INTERIOR) return;
    uint32_t l = i + 1u;
    if (l >= n) return;
    parent[l] = i;
    uint32_t r = nodes[8u * l + 6u];
    if (r > l && r < n) parent[r] = i;
}

// Every parent index is below its child's, so a climb ends within its start
// index; it is also cut at DEPTH_LIMIT.
__global__ void k_blas_depth(const uint32_t* nodes, uint32_t n, const uint32_t* parent, uint32_t* depth) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[8u * i + 7u] == INTERIOR) return;
    uint32_t d = 0, j = i;
    while (parent[j] != NONE && d <= DEPTH_LIMIT) {
        uint32_t p = parent[j];
        if (p >= j) { d = DEPTH_UNKNOWN; break; }
        j = p;
        ++d;
    }
    atomicMax(depth, d > DEPTH_LIMIT ? DEPTH_UNKNOWN : d);
}

__global__ void k_blas_pairs(const uint32_t* nodes, uint32_t n, uint4* pairs) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[8u * i + 7u] != INTERIOR) return;
    uint32_t l = i + 1u;
    uint32_t b0[6] = {0, 0, 0, 0, 0, 0}, b1[6] = {0, 0, 0, 0, 0, 0};
    uint32_t e0 = PE_NONE, e1 = PE_NONE;
    if (l < n) {
        node_box(nodes, l, b0);
        e0 = blas_entry(l, nodes[8u * l + 7u]);
        uint32_t r = nodes[8u * l + 6u];
        if (r > l && r < n) {
            node_box(nodes, r, b1);
            e1 = blas_entry(r, nodes[8u * r + 7u]);
        }
    }
    store_pair(pairs + 4u * i, b0, b1, e0, e1);
}

// One CTA: pair nodes in parallel, then the depth level by level from the root.
constexpr uint32_t TLAS_PAIR_MAX = 2u * PE_TLAS_MAX_SLOTS;

__global__ void __launch_bounds__(1024) k_tlas_pairs(const uint4* tlas, uint32_t n, uint4* pairs, uint32_t* depth) {
    __shared__ uint8_t dep[TLAS_PAIR_MAX];
    __shared__ int changed;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        dep[i] = 0xFFu;
        uint4 b = tlas[2u * i + 1u];
        if ((b.w >> 24) != 0u) continue;  // leaf
        uint32_t l = i + 1u;
        uint32_t b0[6] = {0, 0, 0, 0, 0, 0}, b1[6] = {0, 0, 0, 0, 0, 0};
        uint32_t e0 = PE_NONE, e1 = PE_NONE;
        if (l < n) {
            uint4 la = tlas[2u * l], lb = tlas[2u * l + 1u];
            b0[0] = la.x; b0[1] = la.y; b0[2] = la.z; b0[3] = la.w; b0[4] = lb.x; b0[5] = lb.y;
            e0 = tlas_entry(l, lb.w);
            uint32_t r = lb.z;
            if (r > l && r < n) {
                uint4 ra = tlas[2u * r], rb = tlas[2u * r + 1u];
                b1[0] = ra.x; b1[1] = ra.y; b1[2] = ra.z; b1[3] = ra.w; b1[4] = rb.x; b1[5] = rb.y;
                e1 = tlas_entry(r, rb.w);
            }
        }
        store_pair(pairs + 4u * i, b0, b1, e0, e1);
    }
    __syncthreads();
    if (threadIdx.x == 0) dep[0] = 0;
    uint32_t d = 0;
    for (; d < DEPTH_LIMIT; ++d) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            if (dep[i] != d) continue;
            uint4 b = tlas[2u * i + 1u];
            if ((b.w >> 24) != 0u) continue;
            uint32_t l = i + 1u;
            if (l >= n) continue;
            uint32_t r = tlas[2u * l + 1u].z;
            dep[l] = (uint8_t)(d + 1u);
            if (r > l && r < n) dep[r] = (uint8_t)(d + 1u);
            changed = 1;
        }
        __syncthreads();
        int c = changed;
        __syncthreads();
        if (!c) break;
    }
    if (threadIdx.x == 0) depth[1] = d >= DEPTH_LIMIT ? DEPTH_UNKNOWN : d;
}

}  // namespace

cudaError_t launch_blas_pairs(const SceneBuffers& B, cudaStream_t st) {
    if (!B.pairs || B.nodeCount == 0 || B.nodeCount >= PE_BLAS_MAX_NODES)
        return cudaMemsetAsync(B.depth, 0xFF, 4, st);  // DEPTH_UNKNOWN
    const unsigned g = (B.nodeCount + 255u) / 256u;
    cudaError_t e = cudaMemsetAsync(B.parent, 0xFF, (size_t)B.nodeCount * 4u, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(B.depth, 0, 4, st);
    if (e != cudaSuccess) return e;
    k_blas_link_all<<<g, 256, 0, st>>>(B.nodes, B.nodeCount, B.parent); note_launch();
    k_blas_depth<<<g, 256, 0, st>>>(B.nodes, B.nodeCount, B.parent, B.depth); note_launch();
    k_blas_pairs<<<g, 256, 0, st>>>(B.nodes, B.nodeCount, B.pairs); note_launch();
    return cudaGetLastError();
}

cudaError_t launch_tlas_pairs(const SceneBuffers& B, cudaStream_t st) {
    if (!B.tlasPairs || B.tlasNodeCount == 0 || B.tlasNodeCount > TLAS_PAIR_MAX || B.instCount > PE_TLAS_MAX_SLOTS)
        return cudaMemsetAsync(B.depth + 1, 0xFF, 4, st);  // DEPTH_UNKNOWN
    k_tlas_pairs<<<1, 1024, 0, st>>>(B.tlas, B.tlasNodeCount, B.tlasPairs, B.depth); note_launch();
    return cudaGetLastError();
}

}  // namespace sb
