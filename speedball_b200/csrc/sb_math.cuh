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

// Compensated (Kahan) accumulation s += w * x: the product enters through one
// FMA with the running compensation c, and c keeps the low part that the
// addition to s loses. The compiler does not reassociate these (no fast-math).
__device__ __forceinline__ void kahan_fma(float& s, float& c, float w, float x) {
    const float y = fmaf(w, x, -c);
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// ---- double-float (unevaluated sum hi + lo) arithmetic from FP32 error-free
// transformations (Knuth two-sum, FMA two-product; Dekker 1971). Used where
// FP32 alone would miss the FP64 tolerances: ray angles and the final hit t.
struct dfl { float hi, lo; };
__device__ __forceinline__ dfl two_sum(float a, float b) {
    float s = a + b;
    float bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ dfl fast_two_sum(float a, float b) {
    float s = a + b;
    return {s, b - (s - a)};
}
__device__ __forceinline__ dfl two_prod(float a, float b) {
    float p = a * b;
    return {p, fmaf(a, b, -p)};
}
__device__ __forceinline__ dfl df(float a) { return {a, 0.0f}; }
__device__ __forceinline__ dfl df_add(dfl a, dfl b) {
    dfl s = two_sum(a.hi, b.hi);
    dfl t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dfl df_neg(dfl a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dfl df_sub(dfl a, dfl b) { return df_add(a, df_neg(b)); }
__device__ __forceinline__ dfl df_mul(dfl a, dfl b) {
    dfl p = two_prod(a.hi, b.hi);
    p.lo = fmaf(a.hi, b.lo, fmaf(a.lo, b.hi, p.lo));
    return fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ float df_div(dfl a, dfl b) {
    float q = a.hi / b.hi;
    dfl r = df_sub(a, df_mul(df(q), b));
    return q + r.hi / b.hi;
}
struct df3 { dfl x, y, z; };
__device__ __forceinline__ df3 df3_sub(df3 a, df3 b) { return {df_sub(a.x, b.x), df_sub(a.y, b.y), df_sub(a.z, b.z)}; }
__device__ __forceinline__ dfl df3_dot(df3 a, df3 b) {
    return df_add(df_add(df_mul(a.x, b.x), df_mul(a.y, b.y)), df_mul(a.z, b.z));
}
__device__ __forceinline__ df3 df3_cross(df3 a, df3 b) {
    return {df_sub(df_mul(a.y, b.z), df_mul(a.z, b.y)), df_sub(df_mul(a.z, b.x), df_mul(a.x, b.z)),
            df_sub(df_mul(a.x, b.y), df_mul(a.y, b.x))};
}

// Probe position, gi_probes.js:1714-1726 (relocation x classifyStrength = 0).
__device__ __forceinline__ float3 probe_world_pos(const DevCascade& C, uint32_t p) {
    uint32_t ix = p % C.res[0], iy = (p / C.res[0]) % C.res[1], iz = p / (C.res[0] * C.res[1]);
    float fx = float(ix) / fmaxf(1.0f, float(C.res[0]) - 1.0f);
    float fy = float(iy) / fmaxf(1.0f, float(C.res[1]) - 1.0f);
    float fz = float(iz) / fmaxf(1.0f, float(C.res[2]) - 1.0f);
    return mk(C.gridMin[0] + fx * C.gridSize[0], C.gridMin[1] + fy * C.gridSize[1], C.gridMin[2] + fz * C.gridSize[2]);
}

// Spherical-Fibonacci ray k of N with Cranley-Patterson rotation by the frame
// jitter, normalized (gi_probes.js:1692-1704, 1984, 2331):
//   z = 1 - 2 frac((k + 0.5)/N + j),  phi = k * pi (3 - sqrt 5) + 2 pi j.
// phi reaches hundreds of radians; evaluated naively in FP32 its rounding tilts
// the ray by ~1e-5 rad. Here phi / pi is formed in double-float, reduced mod 2
// exactly and fed to sincospif with a first-order correction for the low part.
// The polar part is double-float too: u = (k + 0.5)/N + j rounded to FP32 moves
// z by ~1e-7, which near the poles (small r) tilts the ray by ~1e-6 rad; with
// u, z and r = sqrt(1 - z^2) = 2 sqrt(u (1 - u)) carried as hi + lo the
// direction keeps ~1e-7 rad of error for every jitter.
__device__ __forceinline__ float3 ray_dir(uint32_t k, uint32_t N, float jitter) {
    const float G_HI = 0.7639320492744446f;       // 3 - sqrt(5) = G_HI + G_LO
    const float G_LO = -2.6774234385129603e-08f;
    const float kk = float(k) + 0.5f, fN = float(N);
    const float q = kk / fN;
    const dfl sk = fast_two_sum(q, fmaf(-q, fN, kk) / fN);  // (k + 0.5) / N, the remainder is exact
    dfl u = df_add(sk, df(jitter));
    float fl = floorf(u.hi);
    if (u.hi == fl && u.lo < 0.0f) fl -= 1.0f;
    const dfl uw = df_add(u, df(-fl));                      // frac, in [0, 1)
    const dfl z = df_add(df(1.0f), dfl{-2.0f * uw.hi, -2.0f * uw.lo});
    // 1 - z^2 = 4 uw (1 - uw); its square root with one Newton step in double-float
    const dfl s4 = df_mul(uw, df_add(df(1.0f), df_neg(uw)));
    float r = 0.0f;
    if (s4.hi > 0.0f) {
        const float r0 = sqrtf(s4.hi);
        const dfl e = df_add(s4, df_neg(two_prod(r0, r0)));
        r = 2.0f * (r0 + (e.hi + e.lo) / (2.0f * r0));
    }
    dfl x = df_add(two_prod(float(k), G_HI), df(float(k) * G_LO));
    x = df_add(x, df(2.0f * jitter));
    float n2 = 2.0f * floorf(x.hi * 0.5f);
    x = df_add(x, df(-n2));
    float s, c;
    sincospif(x.hi, &s, &c);
    float d = 3.141592653589793f * x.lo;
    float s1 = fmaf(c, d, s), c1 = fmaf(-s, d, c);
    return normalize3(mk(r * c1, r * s1, z.hi + z.lo));
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
