// sb_wave.cuh — the per-solve context of the trace wavefront and the shading
// helpers shared by the forward stages (sb_trace.cu) and their adjoint
// (sb_adjoint.cu): hit frame, candidate lights, light gates and terms, sky.
#pragma once
#include "sb_traverse.cuh"

namespace sb {

// The TLAS the walk reads (child pairs when `pairs`, else the 32-byte nodes),
// staged in shared memory when it fits.
__device__ __forceinline__ const uint4* stage_tlas(const WaveCtx& W, uint4* sTlas, bool pairs) {
    const DevScene& S = W.S;
    const uint4* src = pairs ? S.tlasPairs : S.tlas;
    if (W.smemTlas >= S.tlasNodeCount && S.tlasNodeCount > 0) {
        const uint32_t n = (pairs ? 4u : 2u) * S.tlasNodeCount;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sTlas[i] = __ldg(src + i);
        __syncthreads();
        return sTlas;
    }
    return src;
}

struct HitFrame {
    float3 ng, hitPos;
    float traceBias;
    bool faceFwd;
};

// Geometric normal through (M^-1)^T, flipped toward the ray, and the biased
// hit position (gi_probes.js:2003-2017).
__device__ __forceinline__ HitFrame hit_frame(const WaveCtx& W, uint32_t tri, uint32_t inst, float3 ro, float3 rd,
                                              float t, int facing) {
    float4 a = __ldg(W.S.tris + 3 * tri), b = __ldg(W.S.tris + 3 * tri + 1), c = __ldg(W.S.tris + 3 * tri + 2);
    float3 nl = normalize3(cross3(xyz(b) - xyz(a), xyz(c) - xyz(a)));
    float4 r0 = __ldg(W.S.inst + 4 * inst), r1 = __ldg(W.S.inst + 4 * inst + 1), r2 = __ldg(W.S.inst + 4 * inst + 2);
    float3 ngRaw = normalize3(xyz(r0) * nl.x + xyz(r1) * nl.y + xyz(r2) * nl.z);
    HitFrame f;
    f.faceFwd = facing >= 0 ? facing == 1 : dot3(ngRaw, rd) < 0.0f;
    f.ng = ngRaw * (f.faceFwd ? 1.0f : -1.0f);
    f.traceBias = fmaxf(W.C.cellMin * 0.005f * W.P.debugTraceBiasScale, RAY_EPS * W.P.debugRayEpsScale);
    f.hitPos = (ro + rd * t) + f.ng * f.traceBias;
    return f;
}

// Candidate lights of a hit: the C0 cell list in clustered mode
// (gi_probes.js:2109-2127), else every light.
struct LightList {
    const float* list;
    uint32_t count;
};
__device__ __forceinline__ LightList light_list(const WaveCtx& W, float3 hitPos) {
    LightList L{nullptr, W.S.lightCount};
    if (!W.S.clustered) return L;
    const DevCascade& C = W.C;
    float3 cellCount = mk(float(C.g0Res[0]) - 1.0f, float(C.g0Res[1]) - 1.0f, float(C.g0Res[2]) - 1.0f);
    float3 cellSize = mk(C.g0Size[0] / cellCount.x, C.g0Size[1] / cellCount.y, C.g0Size[2] / cellCount.z);
    float3 cf = mk(floorf((hitPos.x - C.g0Min[0]) / cellSize.x), floorf((hitPos.y - C.g0Min[1]) / cellSize.y),
                   floorf((hitPos.z - C.g0Min[2]) / cellSize.z));
    bool outside = cf.x < 0.f || cf.y < 0.f || cf.z < 0.f || cf.x >= cellCount.x || cf.y >= cellCount.y ||
                   cf.z >= cellCount.z;
    uint32_t cx = (uint32_t)clampf(cf.x, 0.f, cellCount.x - 1.0f);
    uint32_t cy = (uint32_t)clampf(cf.y, 0.f, cellCount.y - 1.0f);
    uint32_t cz = (uint32_t)clampf(cf.z, 0.f, cellCount.z - 1.0f);
    uint32_t cellsX = C.g0Res[0] - 1u, cellsY = C.g0Res[1] - 1u;
    uint32_t cellIndex = cz * (cellsX * cellsY) + cy * cellsX + cx;
    const float* list = W.S.lights + LIGHT_DATA + cellIndex * 17u;
    uint32_t listCount = (uint32_t)__ldg(list);
    if (outside || listCount > 16u) return L;
    L.list = list;
    L.count = listCount;
    return L;
}
__device__ __forceinline__ uint32_t light_at(const LightList& L, uint32_t i) {
    return L.list ? (uint32_t)__ldg(L.list + 1 + i) : i;
}

struct LightEval {
    float3 wi, lcol, ldir;
    float dist, ndl, lrange, ldecay, lcosAngle, lcosPen;
    bool isDir, isSpot, pass;
};

// The light record and the gates ahead of the shadow query
// (gi_probes.js:2137-2157 / 2066-2084).
__device__ __forceinline__ LightEval light_eval(const WaveCtx& W, uint32_t li, float3 hitPos, float3 ng) {
    const float* L = W.S.lights + li * 17u;
    LightEval e;
    float ltype = __ldg(L);
    e.pass = false;
    if (!(ltype < 2.5f)) return e;
    float3 lpos = mk(__ldg(L + 1), __ldg(L + 2), __ldg(L + 3));
    e.ldir = mk(__ldg(L + 4), __ldg(L + 5), __ldg(L + 6));
    float eclass = __ldg(L + 16);
    bool isIr = fabsf(eclass - 4.0f) < 0.25f;
    float irs = isIr ? W.P.nirGate * W.P.nirGain : 1.0f;
    e.lcol = mk(__ldg(L + 7), __ldg(L + 8), __ldg(L + 9)) * irs;
    e.lrange = __ldg(L + 10);
    e.ldecay = __ldg(L + 11);
    e.lcosAngle = __ldg(L + 12);
    e.lcosPen = __ldg(L + 13);
    e.isDir = ltype < 0.5f;
    e.isSpot = fabsf(ltype - 2.0f) < 0.5f;
    float3 toLight = e.isDir ? e.ldir * -1.0f : lpos - hitPos;
    e.dist = e.isDir ? 1e4f : fmaxf(sqrtf(dot3(toLight, toLight)), 1e-4f);
    e.wi = normalize3(toLight);
    e.ndl = fmaxf(dot3(ng, e.wi), 0.0f);
    float lpeak = fmaxf(fmaxf(e.lcol.x, e.lcol.y), e.lcol.z);
    e.pass = e.ndl * lpeak > 0.0f && (e.isDir || e.lrange <= 0.0f || e.dist < e.lrange);
    return e;
}

// light_eval's pass decision from the gate table (S.lightGates: the same
// record fields, read as three float4) with the same expressions, so the
// emission stage decides exactly as the shading stage's light_eval.
__device__ __forceinline__ bool light_gate(const WaveCtx& W, uint32_t li, float3 hitPos, float3 ng) {
    const float4 g1 = __ldg(W.S.lightGates + 3u * li + 1u);
    const float ltype = g1.w;
    if (!(ltype < 2.5f)) return false;
    const float4 g0 = __ldg(W.S.lightGates + 3u * li), g2 = __ldg(W.S.lightGates + 3u * li + 2u);
    const bool isIr = fabsf(g2.w - 4.0f) < 0.25f;
    const float irs = isIr ? W.P.nirGate * W.P.nirGain : 1.0f;
    const float3 lcol = xyz(g2) * irs;
    const bool isDir = ltype < 0.5f;
    const float3 toLight = isDir ? xyz(g1) * -1.0f : xyz(g0) - hitPos;
    const float dist = isDir ? 1e4f : fmaxf(sqrtf(dot3(toLight, toLight)), 1e-4f);
    const float3 wi = normalize3(toLight);
    const float ndl = fmaxf(dot3(ng, wi), 0.0f);
    const float lpeak = fmaxf(fmaxf(lcol.x, lcol.y), lcol.z);
    const float lrange = g0.w;
    return ndl * lpeak > 0.0f && (isDir || lrange <= 0.0f || dist < lrange);
}

// The shadow-ray geometry of a light that passed its gates: the direction
// and distance light_eval forms, from the same fields (gate table) and
// expressions.
__device__ __forceinline__ void light_ray(const WaveCtx& W, uint32_t li, float3 hitPos, float3& wi, float& dist) {
    const float4 g1 = __ldg(W.S.lightGates + 3u * li + 1u);
    const bool isDir = g1.w < 0.5f;
    const float3 toLight = isDir ? xyz(g1) * -1.0f : xyz(__ldg(W.S.lightGates + 3u * li)) - hitPos;
    dist = isDir ? 1e4f : fmaxf(sqrtf(dot3(toLight, toLight)), 1e-4f);
    wi = normalize3(toLight);
}

// The unshadowed Lambert NEE term (gi_probes.js:2160-2171).
__device__ __forceinline__ float3 light_term(const WaveCtx& W, const LightEval& e, float3 kd) {
    float falloff = 1.0f / fmaxf(powf(e.dist, e.ldecay), 0.01f);
    float rr = e.dist / fmaxf(e.lrange, 1e-4f);
    float rr2 = rr * rr;
    float win = clampf(1.0f - rr2 * rr2, 0.0f, 1.0f);
    float ranged = falloff * (win * win);
    float posAtten = e.lrange > 0.0f ? ranged : falloff;
    float distAtten = e.isDir ? 1.0f : posAtten;
    float angleCos = dot3(e.wi, e.ldir) * -1.0f;
    float spotAtten = clampf((angleCos - e.lcosAngle) / fmaxf(e.lcosPen - e.lcosAngle, 1e-4f), 0.0f, 1.0f);
    float atten = distAtten * (e.isSpot ? spotAtten : 1.0f);
    float3 diffuse = kd * (1.0f / PI_F);
    return mul3(diffuse * e.ndl, e.lcol) * (atten * W.P.debugDirectScale);
}

__device__ __forceinline__ void ray_of(const WaveCtx& W, uint32_t g, bool dirMajor, uint32_t& slot, uint32_t& k) {
    const uint32_t N = W.C.rays;
    uint32_t s;
    if (dirMajor) {
        k = g / W.slotCount;
        s = g - k * W.slotCount;
        if (W.C.issueOrder) {  // a permutation of every probe (the solve covers them all from slot 0)
            slot = __ldg(W.C.issueOrder + s);
            return;
        }
    } else {
        s = g / N;
        k = g - s * N;
    }
    slot = W.slotBegin + s;
}

// SH-9 sky radiance of a miss (gi_probes.js:2190-2206).
__device__ __forceinline__ float3 sky_sh(const DevParams& P, float3 rd) {
    float x = rd.x, y = rd.y, z = rd.z;
    float b[9] = {0.282095f, y * 0.488603f, z * 0.488603f, x * 0.488603f, x * y * 1.092548f, y * z * 1.092548f,
                  (z * z * 3.0f - 1.0f) * 0.315392f, x * z * 1.092548f, (x * x - y * y) * 0.546274f};
    float3 s = mk(0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 9; ++i) s = s + mk(P.skySH[3 * i], P.skySH[3 * i + 1], P.skySH[3 * i + 2]) * b[i];
    return mk(fmaxf(s.x, 0.f), fmaxf(s.y, 0.f), fmaxf(s.z, 0.f)) * P.skyIntensity;
}

}  // namespace sb
