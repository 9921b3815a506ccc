// sb_math.cuh — small float3 helpers and the per-probe geometry shared by the
// trace and blend kernels (gi_probes.js:1692-1726, gi_oct.js:61-85).
#pragma once
#include "sb_internal.cuh"

namespace sb {

__device__ __forceinline__ float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mul3(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) {
    float l = sqrtf(dot3(a, a));
    return a * (1.0f / l);
}
__device__ __forceinline__ float luma3(float3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

// Probe position, gi_probes.js:1714-1726 (relocation x classifyStrength = 0).
__device__ __forceinline__ float3 probe_world_pos(const DevCascade& C, uint32_t p) {
    uint32_t ix = p % C.res[0], iy = (p / C.res[0]) % C.res[1], iz = p / (C.res[0] * C.res[1]);
    float fx = float(ix) / fmaxf(1.0f, float(C.res[0]) - 1.0f);
    float fy = float(iy) / fmaxf(1.0f, float(C.res[1]) - 1.0f);
    float fz = float(iz) / fmaxf(1.0f, float(C.res[2]) - 1.0f);
    return mk(C.gridMin[0] + fx * C.gridSize[0], C.gridMin[1] + fy * C.gridSize[1], C.gridMin[2] + fz * C.gridSize[2]);
}

// Spherical-Fibonacci ray k of N with Cranley-Patterson rotation by the frame
// jitter, normalized (gi_probes.js:1692-1704, 1984, 2331).
__device__ __forceinline__ float3 ray_dir(uint32_t k, uint32_t N, float jitter) {
    const float GOLDEN = 2.399963229728653f;  // pi * (3 - sqrt(5))
    float sk = (float(k) + 0.5f) / float(N);
    float u = sk + jitter;
    float uw = u - floorf(u);
    float z = 1.0f - uw * 2.0f;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float phi = float(k) * GOLDEN + jitter * 6.283185307179586f;
    float s, c;
    sincosf(phi, &s, &c);
    return normalize3(mk(r * c, r * s, z));
}

// octEncodeNode / octDecodeNode, gi_oct.js:61-85
__device__ __forceinline__ float2 oct_encode(float3 n) {
    float inv = 1.0f / fmaxf(fabsf(n.x) + fabsf(n.y) + fabsf(n.z), 1e-20f);
    float ox = n.x * inv, oy = n.y * inv;
    float fx = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
    float fy = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
    bool lower = n.z < 0.0f;
    float ex = lower ? fx : ox, ey = lower ? fy : oy;
    return make_float2(ex * 0.5f + 0.5f, ey * 0.5f + 0.5f);
}
__device__ __forceinline__ float3 oct_decode(float u, float v) {
    float fx = u * 2.0f - 1.0f, fy = v * 2.0f - 1.0f;
    float nz = 1.0f - fabsf(fx) - fabsf(fy);
    float t = fmaxf(-nz, 0.0f);
    float nx = fx + (fx >= 0.0f ? -t : t);
    float ny = fy + (fy >= 0.0f ? -t : t);
    return normalize3(mk(nx, ny, nz));
}

__device__ __forceinline__ float4 half4_to_float4(uint2 h) {
    __half2 a = *reinterpret_cast<__half2*>(&h.x), b = *reinterpret_cast<__half2*>(&h.y);
    float2 fa = __half22float2(a), fb = __half22float2(b);
    return make_float4(fa.x, fa.y, fb.x, fb.y);
}
__device__ __forceinline__ uint2 float4_to_half4(float4 v) {
    __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
    uint2 r;
    r.x = *reinterpret_cast<uint32_t*>(&a);
    r.y = *reinterpret_cast<uint32_t*>(&b);
    return r;
}

}  // namespace sb
