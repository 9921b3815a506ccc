// sb_pack.cu — validation of the reference wire layouts and the derived
// B200 layouts the traversal reads:
//   * pre-gathered triangles: 3 float4 per triangle (p0 | e1 | e2) with the
//     material's accept bits in p0.w, so a triangle test is three 16-byte
//     loads instead of 3 index + 3 vertex gathers (spectral_traverse.js:390-399);
//   * instance rows: 4 float4 per TLAS slot (3 inverse rows + root/end/sign/active),
//     from the 28-float records (spectral_scene.js:1340-1355);
//   * TLAS nodes: the 12-float records (1356-1365) re-encoded like BLAS nodes
//     (32 bytes, payload (count << 24) | offset).
// Every index the traversal will follow is range-checked here; a violation
// clears the scene's valid word (kernels then do nothing) and latches
// ERR_LAYOUT, which the host reports as SB_ERR_LAYOUT_VIOLATION.
#include "sb_kernels.cuh"

namespace sb {

__device__ __forceinline__ void invalid(uint32_t* valid, uint32_t* err) {
    *valid = 0u;
    latch(err, ERR_LAYOUT);
}

__device__ __forceinline__ bool exact_uint(float f, uint32_t& out) {
    if (!(f >= 0.0f) || !(f < 4294967296.0f) || floorf(f) != f) return false;
    out = (uint32_t)f;
    return true;
}

// Accept bits of one uber record (materialSideAccepts / materialAlphaAccepts /
// traversal flags; spectral_traverse.js:193-222, spectral_scene.js:284-289).
__global__ void k_material_bits(const float* materials, uint32_t materialCount, uint32_t* matBits) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= materialCount) return;
    const float* M = materials + (size_t)m * 28u;
    float side = M[22];
    uint32_t s = side >= 1.5f ? 2u : (side >= 0.5f ? 1u : (side < 0.5f ? 0u : 3u));
    // WGSL u32(f32) of the flags slot; small non-negative integers in practice
    float ff = M[26];
    uint32_t fl = ff > 0.0f ? (uint32_t)ff : 0u;
    float alpha = M[10], alphaTest = M[23];
    bool alphaOk = alpha > 1.0e-4f && (alphaTest <= 0.0f || alpha >= alphaTest);
    bool closest = (fl & 1u) ? alphaOk : ((fl & 2u) != 0u);
    bool shadow = ((fl & 4u) != 0u) && closest;
    matBits[m] = s | (closest ? TB_CLOSEST_OK : 0u) | (shadow ? TB_SHADOW_OK : 0u);
}

__global__ void k_pack_tris(const uint32_t* triIndex, const float* vertexData, const uint32_t* triMaterial,
                            const uint32_t* matBits, uint32_t vertexCount, uint32_t materialCount, uint32_t t0,
                            uint32_t t1, float4* tris, uint32_t* valid, uint32_t* err) {
    uint32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= t1) return;
    uint32_t i0 = triIndex[3 * t], i1 = triIndex[3 * t + 1], i2 = triIndex[3 * t + 2];
    uint32_t m = triMaterial[t];
    if (i0 >= vertexCount || i1 >= vertexCount || i2 >= vertexCount || m >= materialCount) {
        invalid(valid, err);
        return;
    }
    const float* a = vertexData + (size_t)i0 * 8u;
    const float* b = vertexData + (size_t)i1 * 8u;
    const float* c = vertexData + (size_t)i2 * 8u;
    float3 p0 = make_float3(a[0], a[1], a[2]);
    tris[3 * t] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(matBits[m]));
    tris[3 * t + 1] = make_float4(b[0], b[1], b[2], 0.0f);
    tris[3 * t + 2] = make_float4(c[0], c[1], c[2], 0.0f);
}

// Threaded-layout checks that make every BLAS walk memory-safe and finite:
// miss strictly ahead (so a walk advances every step), leaves inside the pool.
__global__ void k_check_nodes(const uint32_t* nodes, uint32_t nodeCount, uint32_t triCount, uint32_t* valid,
                              uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodeCount) return;
    uint32_t miss = nodes[8 * i + 6], payload = nodes[8 * i + 7];
    bool ok = miss > i && miss <= nodeCount;
    if (payload != INTERIOR) {
        uint32_t off = payload & 0x00FFFFFFu, cnt = payload >> 24;
        ok = ok && (uint64_t)off + cnt <= triCount;
    } else {
        ok = ok && i + 1 < nodeCount;
    }
    if (!ok) invalid(valid, err);
}

__global__ void k_pack_instances(const float* materials, uint32_t instBase, uint32_t instCount, uint32_t nodeCount,
                                 float4* inst, uint32_t* valid, uint32_t* err) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= instCount) return;
    const float* R = materials + instBase + (size_t)s * 28u;
    uint32_t root = 0, end = 0;
    float active = R[15];
    bool okRoot = exact_uint(R[12], root), okEnd = exact_uint(R[13], end);
    if (active > 0.5f && !(okRoot && okEnd && root < end && end <= nodeCount)) {
        invalid(valid, err);
        return;
    }
    inst[4 * s] = make_float4(R[0], R[1], R[2], R[3]);
    inst[4 * s + 1] = make_float4(R[4], R[5], R[6], R[7]);
    inst[4 * s + 2] = make_float4(R[8], R[9], R[10], R[11]);
    inst[4 * s + 3] = make_float4(__uint_as_float(root), __uint_as_float(end), R[14], active);
}

__global__ void k_pack_tlas(const float* materials, uint32_t tlasBase, uint32_t tlasNodeCount, uint32_t instCount,
                            uint4* tlas, uint32_t* valid, uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tlasNodeCount) return;
    const float* N = materials + tlasBase + (size_t)i * 12u;
    uint32_t miss = 0, off = 0, cnt = 0;
    bool ok = exact_uint(N[6], miss) && miss > i && miss <= tlasNodeCount;
    float cf = N[8];
    if (cf >= 0.5f) {
        // instCountF >= 0.5 descends into uint(instCountF) instances from uint(off)
        cnt = (uint32_t)cf;
        ok = ok && exact_uint(N[7], off) && cnt < 256u && off < (1u << 24) && (uint64_t)off + cnt <= instCount;
    } else {
        cnt = 0;
        ok = ok && i + 1 < tlasNodeCount;
    }
    if (!ok) {
        invalid(valid, err);
        return;
    }
    tlas[2 * i] = make_uint4(__float_as_uint(N[0]), __float_as_uint(N[1]), __float_as_uint(N[2]), __float_as_uint(N[3]));
    tlas[2 * i + 1] = make_uint4(__float_as_uint(N[4]), __float_as_uint(N[5]), miss, (cnt << 24) | off);
}

static inline unsigned blocks(uint32_t n, unsigned b) { return (n + b - 1) / b; }

cudaError_t launch_pack_tris(const SceneBuffers& B, uint32_t t0, uint32_t t1, uint32_t* err, cudaStream_t st) {
    if (t1 > t0) {
        k_pack_tris<<<blocks(t1 - t0, 256), 256, 0, st>>>(B.triIndex, B.vertexData, B.triMaterial, B.matBits,
                                                          B.vertexCount, B.materialCount, t0, t1, B.tris, B.valid, err);
        note_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_pack_dynamic(const SceneBuffers& B, uint32_t* err, cudaStream_t st) {
    if (B.instCount) {
        k_pack_instances<<<blocks(B.instCount, 128), 128, 0, st>>>(B.materials, B.instBase, B.instCount, B.nodeCount,
                                                                   B.inst, B.valid, err);
        note_launch();
    }
    if (B.tlasNodeCount) {
        k_pack_tlas<<<blocks(B.tlasNodeCount, 128), 128, 0, st>>>(B.materials, B.tlasBase, B.tlasNodeCount,
                                                                  B.instCount, B.tlas, B.valid, err);
        note_launch();
    }
    cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : launch_tlas_pairs(B, st);
}

cudaError_t launch_pack_scene(const SceneBuffers& B, uint32_t* err, cudaStream_t st) {
    if (B.materialCount) {
        k_material_bits<<<blocks(B.materialCount, 128), 128, 0, st>>>(B.materials, B.materialCount, B.matBits);
        note_launch();
    }
    if (B.nodeCount) {
        k_check_nodes<<<blocks(B.nodeCount, 256), 256, 0, st>>>(B.nodes, B.nodeCount, B.triCount, B.valid, err);
        note_launch();
    }
    cudaError_t e = launch_blas_pairs(B, st);
    if (e != cudaSuccess) return e;
    e = launch_pack_tris(B, 0, B.triCount, err, st);
    if (e != cudaSuccess) return e;
    return launch_pack_dynamic(B, err, st);
}

}  // namespace sb
