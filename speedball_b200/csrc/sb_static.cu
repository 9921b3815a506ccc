// sb_static.cu — BLAS refit that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host whose device memory is owned by
// another allocator (a renderer's interop heap that hands out only its own
// buffers), or a per-frame path that must not allocate because cudaMalloc can
// synchronize the whole device and stall the frame. This entry point serves
// them. The caller passes its own device buffers (nodes in/out, triangle
// indices, vertices); the refit's scratch (parent links, arrival counters, the
// layout gate) lives in one file-scope device array below, sized at build time.
//
// The array is shared by every call on a device and keeps the last call's
// contents; each call clears the part it uses. Calls that overlap on the GPU
// (two host threads, or two streams, refitting at once) race on it.
// Every call resolves the array's device address (cudaGetSymbolAddress) with
// the device current; the first call on a device may load the library's device
// code there, so make it before any stream capture.
#include <cstdio>
#include <cstring>

#include "sb_kernels.cuh"

namespace {

constexpr uint32_t kMaxNodes = SB_REFIT_STATIC_MAX_NODES;
constexpr uint32_t NONE = 0xFFFFFFFFu;

// [0, kMaxNodes) parent links, [kMaxNodes, 2*kMaxNodes) arrival counters,
// [2*kMaxNodes] layout gate (1 = valid).
static __device__ __align__(256) uint32_t g_refitScratch[2 * kMaxNodes + 64];

__global__ void k_static_reset(uint32_t* scratch, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        scratch[i] = NONE;
        scratch[kMaxNodes + i] = 0u;
    }
    if (i == 0) scratch[2 * kMaxNodes] = 1u;
}

// Layout contract of refitFlatBlasRange (gi_refit.js:96-139): right child =
// left child's miss inside (left, end); leaves inside the pools.
__global__ void k_static_link(const uint32_t* nodes, const uint32_t* triIndex, uint32_t triCount,
                              uint32_t vertexCount, uint32_t* scratch, uint32_t root, uint32_t end) {
    uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    uint32_t* gate = scratch + 2 * kMaxNodes;
    uint32_t info = nodes[8 * i + 7];
    if (info != sb::INTERIOR) {
        uint32_t off = info & 0x00FFFFFFu, cnt = info >> 24;
        for (uint32_t t = off; t < off + cnt; ++t) {
            if (t >= triCount) { *gate = 0u; return; }
            for (int k = 0; k < 3; ++k)
                if (triIndex[3 * t + k] >= vertexCount) { *gate = 0u; return; }
        }
        return;
    }
    uint32_t l = i + 1;
    if (l >= end) { *gate = 0u; return; }
    uint32_t r = nodes[8 * l + 6];
    if (!(r > l && r < end)) { *gate = 0u; return; }
    if (atomicCAS(&scratch[l - root], NONE, i) != NONE) *gate = 0u;
    if (atomicCAS(&scratch[r - root], NONE, i) != NONE) *gate = 0u;
}

__global__ void k_static_orphans(const uint32_t* scratch_ro, uint32_t* scratch, uint32_t root, uint32_t end) {
    uint32_t i = root + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    if (scratch_ro[i - root] == NONE) scratch[2 * kMaxNodes] = 0u;
}

__device__ __forceinline__ float vload(const uint32_t* p) { return __uint_as_float(*(const volatile uint32_t*)p); }

// Exact leaf min/max in the reference's order, then the second child to finish
// unions its parent (JS Math.min/max), up to the root.
__global__ void k_static_run(uint32_t* nodes, const uint32_t* triIndex, const float* vertexData, uint32_t* scratch,
                             uint32_t root, uint32_t end) {
    uint32_t i = root + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end || *(volatile uint32_t*)&scratch[2 * kMaxNodes] == 0u) return;
    uint32_t info = nodes[8 * i + 7];
    if (info == sb::INTERIOR) return;
    uint32_t off = info & 0x00FFFFFFu, cnt = info >> 24;
    if (cnt != 0u) {
        float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
        for (uint32_t t = off; t < off + cnt; ++t)
            for (int k = 0; k < 3; ++k) {
                const float* v = vertexData + (size_t)triIndex[3 * t + k] * 8u;
                float x = v[0], y = v[1], z = v[2];
                if (x < mnx) mnx = x;
                if (x > mxx) mxx = x;
                if (y < mny) mny = y;
                if (y > mxy) mxy = y;
                if (z < mnz) mnz = z;
                if (z > mxz) mxz = z;
            }
        uint32_t* n = nodes + 8 * i;
        n[0] = __float_as_uint(mnx); n[1] = __float_as_uint(mny); n[2] = __float_as_uint(mnz);
        n[3] = __float_as_uint(mxx); n[4] = __float_as_uint(mxy); n[5] = __float_as_uint(mxz);
    }
    uint32_t node = i;
    for (;;) {
        uint32_t p = scratch[node - root];
        if (p == NONE) break;
        __threadfence();
        if (atomicAdd(&scratch[kMaxNodes + (p - root)], 1u) == 0u) break;
        __threadfence();
        uint32_t l = p + 1;
        uint32_t r = *(const volatile uint32_t*)(nodes + 8 * l + 6);
        const uint32_t* L = nodes + 8 * l;
        const uint32_t* R = nodes + 8 * r;
        uint32_t* n = nodes + 8 * p;
        n[0] = __float_as_uint(sb::js_min(vload(L + 0), vload(R + 0)));
        n[1] = __float_as_uint(sb::js_min(vload(L + 1), vload(R + 1)));
        n[2] = __float_as_uint(sb::js_min(vload(L + 2), vload(R + 2)));
        n[3] = __float_as_uint(sb::js_max(vload(L + 3), vload(R + 3)));
        n[4] = __float_as_uint(sb::js_max(vload(L + 4), vload(R + 4)));
        n[5] = __float_as_uint(sb::js_max(vload(L + 5), vload(R + 5)));
        node = p;
    }
}

void put_msg(char* msg, size_t len, const char* text) {
    if (msg && len) {
        std::strncpy(msg, text, len - 1);
        msg[len - 1] = '\0';
    }
}

}  // namespace

extern "C" sb_status sb_refit_blas_static(uint32_t* nodes, uint32_t nodeCount, const uint32_t* triIndex,
                                          uint32_t triCount, const float* vertexData, uint32_t vertexCount,
                                          uint32_t root, uint32_t end, void* cudaStream, char* msg, size_t msgLen) {
    if (!nodes || !triIndex || !vertexData) {
        put_msg(msg, msgLen, "sb_refit_blas_static: null device pointer");
        return SB_ERR_INVALID_ARG;
    }
    if (!(end > root && end <= nodeCount)) {
        put_msg(msg, msgLen, "sb_refit_blas_static: node range outside the pool");
        return SB_ERR_LAYOUT_VIOLATION;
    }
    if (end - root > kMaxNodes) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "sb_refit_blas_static: %u nodes exceed the static scratch maximum of %u nodes",
                      end - root, kMaxNodes);
        put_msg(msg, msgLen, buf);
        return SB_ERR_INVALID_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        put_msg(msg, msgLen, "sb_refit_blas_static: no current CUDA device");
        return SB_ERR_NO_DEVICE;
    }
    // The host-side name of a __device__ array is not a device address: look
    // the address up with the device current. Every call looks it up again (a
    // lookup, no allocation), so an address cached across a cudaDeviceReset,
    // after which the module and its array are loaded anew, is never used.
    void* sym = nullptr;
    cudaError_t se = cudaGetSymbolAddress(&sym, g_refitScratch);
    if (se != cudaSuccess || !sym) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "sb_refit_blas_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(se));
        put_msg(msg, msgLen, buf);
        return SB_ERR_CUDA;
    }
    uint32_t* scratch = static_cast<uint32_t*>(sym);
    cudaStream_t st = (cudaStream_t)cudaStream;
    const uint32_t n = end - root;
    const unsigned g = (n + 255) / 256;
    k_static_reset<<<g, 256, 0, st>>>(scratch, n);
    k_static_link<<<g, 256, 0, st>>>(nodes, triIndex, triCount, vertexCount, scratch, root, end);
    k_static_orphans<<<g, 256, 0, st>>>(scratch, scratch, root, end);
    k_static_run<<<g, 256, 0, st>>>(nodes, triIndex, vertexData, scratch, root, end);
    for (int k = 0; k < 4; ++k) sb::note_launch();
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        put_msg(msg, msgLen, cudaGetErrorString(le));
        return SB_ERR_CUDA;
    }
    uint32_t gate = 0;
    cudaError_t e = cudaMemcpyAsync(&gate, scratch + 2 * kMaxNodes, sizeof gate, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        put_msg(msg, msgLen, cudaGetErrorString(e));
        return SB_ERR_CUDA;
    }
    if (!gate) {
        put_msg(msg, msgLen, "sb_refit_blas_static: threaded-layout violation (full rebuild required)");
        return SB_ERR_LAYOUT_VIOLATION;
    }
    put_msg(msg, msgLen, "");
    return SB_OK;
}
