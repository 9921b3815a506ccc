// sb_build.cu — BLAS build on the GPU in the reference's threaded layout.
//
// The reference builds each BLAS on the CPU with three-mesh-bvh
// (spectral_scene.js:898-966, ~200 ms for a large mesh, the cost its refit
// lane exists to avoid, gi_refit.js:7-8) and re-flattens it into 8 x u32
// nodes (flattenBVHRoot, 658-721). This builder is a linear BVH (Karras,
// "Maximizing Parallelism in the Construction of BVHs, Octrees, and k-d
// Trees", HPG 2012) emitting that layout directly:
//   1. per triangle its vertex bounds; the centroid bounds of the mesh;
//   2. a 30-bit Morton code of each bounds centre within the centroid bounds;
//   3. a stable LSD radix sort of (code, triangle), 4 passes of 8 bits, with
//      warp-level ranking (match.any) so equal digits keep their order;
//   4. the binary radix tree over the sorted codes, equal codes ordered by
//      position (Karras' tie rule), one thread per internal node;
//   5. a bottom-up pass (one thread per triangle, arrival counters: the second
//      child to arrive carries on) giving every node its bounds (exact min/max
//      of its triangles' vertices, as the refit computes them) and its size in
//      the output tree, where any node of at most `leafSize` triangles whose
//      parent holds more becomes one leaf;
//   6. every output node finds its pre-order index by walking to the root
//      (adding 1 per ancestor and, when it lies right of an ancestor, the size
//      of that ancestor's left subtree) and writes its record: bounds, miss =
//      index + subtree size, payload (count << 24 | first position) or
//      0xFFFFFFFF. The left child lands at index + 1.
// The output triangle order is the sorted order (triangle at each position).
// No loop waits on another thread; every walk is bounded by the tree depth
// (at most 64 levels: each level adds a bit of the 62-bit key + position).
#include "sb_kernels.cuh"

namespace sb {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kTile = 2048;   // keys per sort CTA (8 warps x 8 rounds x 32)
constexpr uint32_t kSortThreads = 256;

__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 1. triangle bounds (source order) and the centroid bounds
__global__ void k_tri_bounds(const float* pos, uint32_t V, const uint32_t* idx, uint32_t T, float4* lo, float4* hi,
                             uint32_t* cbox, uint32_t* err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {0.f, 0.f, 0.f};
    bool valid = false;
    if (t < T) {
        const uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
        if (i0 < V && i1 < V && i2 < V) {
            float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
            const uint32_t ids[3] = {i0, i1, i2};
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) {
                    const float v = pos[3 * (size_t)ids[k] + a];
                    if (v < mn[a]) mn[a] = v;
                    if (v > mx[a]) mx[a] = v;
                }
            lo[t] = make_float4(mn[0], mn[1], mn[2], 0.0f);
            hi[t] = make_float4(mx[0], mx[1], mx[2], 0.0f);
            for (int a = 0; a < 3; ++a) c[a] = mn[a] + (mx[a] - mn[a]) * 0.5f;
            valid = isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]);
        } else {
            latch(err, ERR_LAYOUT);
            lo[t] = make_float4(0.f, 0.f, 0.f, 0.f);
            hi[t] = lo[t];
        }
    }
    // warp-reduce the ordered-int centroid bounds, one atomic per warp and bound
    uint32_t omn[3], omx[3];
    for (int a = 0; a < 3; ++a) {
        omn[a] = valid ? f2o(c[a]) : 0xFFFFFFFFu;
        omx[a] = valid ? f2o(c[a]) : 0u;
        for (int s = 16; s; s >>= 1) {
            omn[a] = min(omn[a], __shfl_xor_sync(0xFFFFFFFFu, omn[a], s));
            omx[a] = max(omx[a], __shfl_xor_sync(0xFFFFFFFFu, omx[a], s));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(cbox + a, omn[a]);
            atomicMax(cbox + 3 + a, omx[a]);
        }
}

// 2. Morton codes of the bounds centres
__global__ void k_morton(const float4* lo, const float4* hi, uint32_t T, const uint32_t* cbox, uint32_t* keys,
                         uint32_t* vals) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const float4 l = lo[t], h = hi[t];
    const float c[3] = {l.x + (h.x - l.x) * 0.5f, l.y + (h.y - l.y) * 0.5f, l.z + (h.z - l.z) * 0.5f};
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float mn = o2f(cbox[a]), mx = o2f(cbox[3 + a]);
        const float ext = mx - mn;
        float x = ext > 0.0f ? (c[a] - mn) / ext : 0.0f;
        x = isfinite(x) ? fminf(fmaxf(x, 0.0f), 1.0f) : 0.0f;
        q[a] = min((uint32_t)(x * 1024.0f), 1023u);
    }
    keys[t] = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
    vals[t] = t;
}

// 3. stable LSD radix sort, one 8-bit digit per pass
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const uint32_t* keys, uint32_t T, uint32_t shift,
                                                            uint32_t* hist, uint32_t tiles) {
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t base = blockIdx.x * kTile;
    for (uint32_t i = threadIdx.x; i < kTile; i += kSortThreads) {
        const uint32_t p = base + i;
        if (p < T) atomicAdd(&cnt[(keys[p] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of n counts in place, one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_scan(uint32_t* a, uint32_t n) {
    __shared__ uint32_t warpSum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? a[i] : 0u;
        uint32_t x = v;
        for (int s = 1; s < 32; s <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, s);
            if (lane >= (uint32_t)s) x += y;
        }
        if (lane == 31) warpSum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = warpSum[lane];
            for (int k = 1; k < 32; k <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, k);
                if (lane >= (uint32_t)k) s += y;
            }
            warpSum[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = (w ? warpSum[w - 1] : 0u) + x - v;
        if (i < n) a[i] = carry + before;
        __syncthreads();
        if (threadIdx.x == 1023) carry += warpSum[31];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const uint32_t* keysIn, const uint32_t* valsIn,
                                                               uint32_t T, uint32_t shift, const uint32_t* hist,
                                                               uint32_t tiles, uint32_t* keysOut,
                                                               uint32_t* valsOut) {
    __shared__ uint32_t warpCnt[8][256];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t d = lane; d < 256; d += 32) warpCnt[w][d] = 0u;
    __syncwarp();
    const uint32_t seg = blockIdx.x * kTile + w * 256u;
    const uint32_t ltMask = (1u << lane) - 1u;
    uint32_t key[8], val[8], rank[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t p = seg + (uint32_t)k * 32u + lane;
        const bool valid = p < T;
        key[k] = valid ? keysIn[p] : 0u;
        val[k] = valid ? valsIn[p] : 0u;
        const uint32_t digit = (key[k] >> shift) & 0xFFu;
        const uint32_t tag = valid ? digit : 0x100u;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, tag);
        const uint32_t base = valid ? warpCnt[w][digit] : 0u;
        __syncwarp();
        if (valid && lane == (uint32_t)(__ffs(peers) - 1)) warpCnt[w][digit] = base + __popc(peers);
        __syncwarp();
        rank[k] = base + __popc(peers & ltMask);
    }
    __syncthreads();
    // per digit: offsets of the warps in position order
    {
        const uint32_t d = threadIdx.x;
        uint32_t run = 0u;
        for (int ww = 0; ww < 8; ++ww) {
            const uint32_t c = warpCnt[ww][d];
            warpCnt[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t p = seg + (uint32_t)k * 32u + lane;
        if (p >= T) continue;
        const uint32_t digit = (key[k] >> shift) & 0xFFu;
        const uint32_t dst = hist[digit * tiles + blockIdx.x] + warpCnt[w][digit] + rank[k];
        keysOut[dst] = key[k];
        valsOut[dst] = val[k];
    }
}

// 4. binary radix tree (internal nodes 0..T-2, leaf j = T-1+j)
__device__ __forceinline__ int delta(const uint32_t* keys, int64_t T, int64_t i, int64_t j) {
    if (j < 0 || j >= T) return -1;
    const uint32_t a = keys[i], b = keys[j];
    if (a == b) return __clzll((unsigned long long)(i ^ j));  // >= 32 for positions below 2^32
    return __clz(a ^ b);
}

__global__ void k_radix_tree(const uint32_t* keys, uint32_t T, uint32_t* parent, uint32_t* left, uint32_t* right,
                             uint32_t* first, uint32_t* last, uint32_t* err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n = T;
    if (i >= n - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int64_t lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int64_t s = 0;
    for (int64_t div = 2;; div *= 2) {
        const int64_t t = (l + div - 1) / div;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int64_t g = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = i < j ? i : j, hiR = i < j ? j : i;
    if (!(lo <= g && g < hiR && hiR < n)) {  // the split lies inside the node's range
        latch(err, ERR_LAYOUT);
        left[i] = right[i] = kNone;
        first[i] = last[i] = (uint32_t)i;
        return;
    }
    const uint32_t L = (lo == g) ? (uint32_t)(n - 1 + g) : (uint32_t)g;
    const uint32_t R = (hiR == g + 1) ? (uint32_t)(n - 1 + g + 1) : (uint32_t)(g + 1);
    left[i] = L;
    right[i] = R;
    first[i] = (uint32_t)lo;
    last[i] = (uint32_t)hiR;
    parent[L] = (uint32_t)i;
    parent[R] = (uint32_t)i;
    if (i == 0) parent[0] = kNone;
}

struct Tree {
    uint32_t T, leafSize;
    const uint32_t *parent, *left, *right, *first, *last, *vals;
    const float4 *triLo, *triHi;
    float4 *boxLo, *boxHi;
    uint32_t* size;
    uint32_t* arrive;
    const float* pos;      // source vertices, 3 floats each
    const uint32_t* idx;   // source triangles, 3 indices each
};

// A leaf's bounds exactly as the refit computes them (gi_refit.js:108-113):
// its triangles in BVH order, their vertices in index order, strict < / >
// updates (so the sign of a zero bound matches the refit's).
__device__ __forceinline__ void leaf_bounds(const Tree& R, uint32_t f, uint32_t l, float4& lo, float4& hi) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t q = f; q <= l; ++q) {
        const uint32_t t = R.vals[q];
        for (int k = 0; k < 3; ++k) {
            const float* v = R.pos + 3 * (size_t)R.idx[3 * (size_t)t + k];
            for (int a = 0; a < 3; ++a) {
                if (v[a] < mn[a]) mn[a] = v[a];
                if (v[a] > mx[a]) mx[a] = v[a];
            }
        }
    }
    lo = make_float4(mn[0], mn[1], mn[2], 0.0f);
    hi = make_float4(mx[0], mx[1], mx[2], 0.0f);
}

__device__ __forceinline__ uint32_t count_of(const Tree& R, uint32_t node) {
    return node < R.T - 1 ? R.last[node] - R.first[node] + 1u : 1u;
}

// 5. bottom-up: bounds and output sizes
__global__ void k_climb(Tree R, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= R.T) return;
    uint32_t node = R.T - 1 + j;
    for (int level = 0;; ++level) {
        const uint32_t p = R.parent[node];
        if (p == kNone) break;
        if (level >= 80) {  // deeper than any radix tree of 32-bit codes and positions
            latch(err, ERR_LAYOUT);
            break;
        }
        uint32_t prev;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(R.arrive + p) : "memory");
        if (prev == 0u) break;
        const uint32_t L = R.left[p], Rt = R.right[p];
        if (p >= R.T - 1 || L >= 2 * R.T - 1 || Rt >= 2 * R.T - 1) {
            latch(err, ERR_LAYOUT);
            break;
        }
        float4 ll, lh, rl, rh;
        uint32_t sl, sr;
        if (L < R.T - 1) {
            ll = __ldcg(R.boxLo + L); lh = __ldcg(R.boxHi + L); sl = __ldcg(R.size + L);
        } else {
            const uint32_t t = R.vals[L - (R.T - 1)];
            ll = R.triLo[t]; lh = R.triHi[t]; sl = 1u;
        }
        if (Rt < R.T - 1) {
            rl = __ldcg(R.boxLo + Rt); rh = __ldcg(R.boxHi + Rt); sr = __ldcg(R.size + Rt);
        } else {
            const uint32_t t = R.vals[Rt - (R.T - 1)];
            rl = R.triLo[t]; rh = R.triHi[t]; sr = 1u;
        }
        if (count_of(R, p) <= R.leafSize) {  // one output leaf: bounds as the refit's leaf rule
            float4 lo, hi;
            leaf_bounds(R, R.first[p], R.last[p], lo, hi);
            R.boxLo[p] = lo;
            R.boxHi[p] = hi;
            R.size[p] = 1u;
        } else {                             // an interior node: the refit's union of its two children
            R.boxLo[p] = make_float4(js_min(ll.x, rl.x), js_min(ll.y, rl.y), js_min(ll.z, rl.z), 0.0f);
            R.boxHi[p] = make_float4(js_max(lh.x, rh.x), js_max(lh.y, rh.y), js_max(lh.z, rh.z), 0.0f);
            R.size[p] = 1u + sl + sr;
        }
        node = p;
    }
}

// 6. pre-order index and record of every output node
__global__ void k_emit_nodes(Tree R, uint32_t* nodes, uint32_t* nodeCount, uint32_t* err) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= 2 * R.T - 1) return;
    const uint32_t p0 = R.parent[x];
    // emitted: the root, and every node whose parent is interior in the output
    if (p0 != kNone && count_of(R, p0) <= R.leafSize) return;
    uint32_t idx = 0u, c = x;
    for (int level = 0;; ++level) {
        const uint32_t a = R.parent[c];
        if (a == kNone) break;
        if (level >= 80) {
            latch(err, ERR_LAYOUT);
            return;
        }
        if (a >= R.T - 1) {
            latch(err, ERR_LAYOUT);
            return;
        }
        idx += 1u;
        if (R.right[a] == c) {
            const uint32_t L = R.left[a];
            idx += L < R.T - 1 ? R.size[L] : 1u;
        }
        c = a;
    }
    const bool internal = x < R.T - 1;
    float4 lo, hi;
    uint32_t sz, payload;
    if (internal) {
        lo = R.boxLo[x];
        hi = R.boxHi[x];
        sz = R.size[x];
        const uint32_t cnt = count_of(R, x);
        payload = cnt <= R.leafSize ? ((cnt << 24) | R.first[x]) : 0xFFFFFFFFu;
    } else {
        const uint32_t j = x - (R.T - 1), t = R.vals[j];
        lo = R.triLo[t];
        hi = R.triHi[t];
        sz = 1u;
        payload = (1u << 24) | j;
    }
    if ((uint64_t)idx + sz > 2ull * R.T - 1ull) {  // sizes that do not add up: never write outside
        latch(err, ERR_LAYOUT);
        return;
    }
    uint32_t* n = nodes + 8ull * idx;
    n[0] = __float_as_uint(lo.x); n[1] = __float_as_uint(lo.y); n[2] = __float_as_uint(lo.z);
    n[3] = __float_as_uint(hi.x); n[4] = __float_as_uint(hi.y); n[5] = __float_as_uint(hi.z);
    n[6] = idx + sz;
    n[7] = payload;
    if (p0 == kNone) *nodeCount = sz;
}

template <class Tp> cudaError_t grow(Tp*& p, size_t& cap, size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, n * sizeof(Tp));
    if (e == cudaSuccess) cap = n;
    return e;
}

}  // namespace

struct BlasBuilder {
    float4 *triLo = nullptr, *triHi = nullptr, *boxLo = nullptr, *boxHi = nullptr;
    uint32_t *keyA = nullptr, *keyB = nullptr, *valA = nullptr, *valB = nullptr, *hist = nullptr;
    uint32_t *cbox = nullptr, *parent = nullptr, *left = nullptr, *right = nullptr, *first = nullptr,
             *last = nullptr, *arrive = nullptr, *size = nullptr;
    size_t cT = 0, cT2 = 0, cK = 0, cH = 0, cN = 0, cBox = 0, cI = 0, cI2 = 0, cC = 0;
    size_t cA = 0, cB = 0, cV = 0, cW = 0, cP = 0, cL = 0, cR = 0, cF = 0, cLa = 0, cAr = 0, cS = 0;

    cudaError_t reserve(uint32_t T) {
        const size_t tiles = (T + kTile - 1) / kTile;
        cudaError_t e = cudaSuccess;
        if (e == cudaSuccess) e = grow(triLo, cT, T);
        if (e == cudaSuccess) e = grow(triHi, cT2, T);
        if (e == cudaSuccess) e = grow(boxLo, cBox, T);
        if (e == cudaSuccess) e = grow(boxHi, cN, T);
        if (e == cudaSuccess) e = grow(keyA, cA, T);
        if (e == cudaSuccess) e = grow(keyB, cB, T);
        if (e == cudaSuccess) e = grow(valA, cV, T);
        if (e == cudaSuccess) e = grow(valB, cW, T);
        if (e == cudaSuccess) e = grow(hist, cH, 256 * tiles);
        if (e == cudaSuccess) e = grow(cbox, cC, 6);
        if (e == cudaSuccess) e = grow(parent, cP, 2 * (size_t)T);
        if (e == cudaSuccess) e = grow(left, cL, T);
        if (e == cudaSuccess) e = grow(right, cR, T);
        if (e == cudaSuccess) e = grow(first, cF, T);
        if (e == cudaSuccess) e = grow(last, cLa, T);
        if (e == cudaSuccess) e = grow(arrive, cAr, T);
        if (e == cudaSuccess) e = grow(size, cS, T);
        return e;
    }
    ~BlasBuilder() {
        for (void* p : {(void*)triLo, (void*)triHi, (void*)boxLo, (void*)boxHi, (void*)keyA, (void*)keyB,
                        (void*)valA, (void*)valB, (void*)hist, (void*)cbox, (void*)parent, (void*)left,
                        (void*)right, (void*)first, (void*)last, (void*)arrive, (void*)size})
            if (p) cudaFree(p);
    }
};

BlasBuilder* blas_builder_create() { return new BlasBuilder(); }
void blas_builder_destroy(BlasBuilder* b) { delete b; }

cudaError_t blas_build(BlasBuilder* b, const float* pos, uint32_t V, const uint32_t* idx, uint32_t T,
                       uint32_t leafSize, uint32_t* nodes, uint32_t* order, uint32_t* nodeCount, uint32_t* err,
                       cudaStream_t st) {
    if (T == 0) return cudaSuccess;
    cudaError_t e = b->reserve(T);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (T + kTile - 1) / kTile;
    const unsigned g = (T + 255) / 256;
    // centroid bounds start empty: min words at the largest ordered value, max at 0
    if ((e = cudaMemsetAsync(b->cbox, 0xFF, 3 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b->cbox + 3, 0, 3 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    k_tri_bounds<<<g, 256, 0, st>>>(pos, V, idx, T, b->triLo, b->triHi, b->cbox, err); note_launch();
    k_morton<<<g, 256, 0, st>>>(b->triLo, b->triHi, T, b->cbox, b->keyA, b->valA); note_launch();
    uint32_t *kin = b->keyA, *vin = b->valA, *kout = b->keyB, *vout = b->valB;
    for (uint32_t shift = 0; shift < 32; shift += 8) {
        k_sort_hist<<<tiles, kSortThreads, 0, st>>>(kin, T, shift, b->hist, tiles); note_launch();
        k_scan<<<1, 1024, 0, st>>>(b->hist, 256 * tiles); note_launch();
        k_sort_scatter<<<tiles, kSortThreads, 0, st>>>(kin, vin, T, shift, b->hist, tiles, kout, vout); note_launch();
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    // after 4 passes the sorted keys and triangles are back in keyA / valA
    if ((e = cudaMemcpyAsync(order, vin, (size_t)T * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    if (T == 1) {
        // one triangle: the root is a leaf
        Tree R{T, leafSize, b->parent, b->left, b->right, b->first, b->last, vin, b->triLo, b->triHi, b->boxLo,
               b->boxHi, b->size, b->arrive, pos, idx};
        if ((e = cudaMemsetAsync(b->parent, 0xFF, sizeof(uint32_t), st)) != cudaSuccess) return e;  // no parent
        k_emit_nodes<<<1, 32, 0, st>>>(R, nodes, nodeCount, err); note_launch();
        return cudaGetLastError();
    }
    if ((e = cudaMemsetAsync(b->arrive, 0, (size_t)(T - 1) * 4, st)) != cudaSuccess) return e;
    k_radix_tree<<<(T - 1 + 255) / 256, 256, 0, st>>>(kin, T, b->parent, b->left, b->right, b->first, b->last, err);
    note_launch();
    Tree R{T, leafSize, b->parent, b->left, b->right, b->first, b->last, vin, b->triLo, b->triHi, b->boxLo,
           b->boxHi, b->size, b->arrive, pos, idx};
    k_climb<<<g, 256, 0, st>>>(R, err); note_launch();
    k_emit_nodes<<<(2 * T - 1 + 255) / 256, 256, 0, st>>>(R, nodes, nodeCount, err); note_launch();
    return cudaGetLastError();
}

}  // namespace sb
