// sb_gather.cu — the receiver gather: the irradiance the probe field gives a
// surface point, the consumer of the atlases this library updates. The
// reference evaluates it per fragment in GiProbeNode (gi_probes.js:530-657,
// 816-850, 884-928); here one thread evaluates one G-buffer sample.
//
// Per sample: P = position * samplePositionScale + Nvis * normalBias[0] *
// sampleBiasScale; with one cascade, _sampleCascade at P; with two, the coarse
// and fine looped gathers blended by the fine box's border band, each choosing
// its cage at the unbiased surface position (the looped gather's stated intent,
// gi_probes.js:628-631). Each of the 8 cage taps fetches the RGBA16F atlas
// bilinearly (exact weights; the footprint stays inside the probe's tile, so the
// sampler's edge clamp never applies) in the detail normal's octahedral
// direction; with chebyStrength > 0 it also fetches the depth moments toward
// the surface for the Chebyshev visibility weight and applies the wrap weight.
// Output E = max(sample, 0) * intensity * enabled as float4 (rgb, 1).
//
// Work is one probe field's worth of tiny atlases (L1/L2-resident) against a
// streamed G-buffer: 48 bytes in and 16 bytes out per sample are the HBM
// traffic, so the kernel is HBM-bound on the G-buffer stream. Classification
// is inert (classifyStrength 0): no state atlas is read.
#include "sb_kernels.cuh"
#include "sb_math.cuh"

namespace sb {

namespace {

// A bilinear read inside one probe's octahedral tile. The atlas coordinate of
// direction o is tileOrigin + BORDER + o * octRes - 0.5 (texel centres), so the
// tile-local coordinate 0.5 + o * octRes lies in [0.5, octRes + 0.5]: the 2x2
// footprint never leaves the tile (gutter included), edge clamping never
// applies, and the offset and weights are the same for every tap that reads the
// same direction. Formed once, without the atlas-wide coordinate's rounding.
struct TileTap {
    uint32_t off;  // first texel of the footprint, from the tile origin (row * W + column)
    float fx, fy;
};
__device__ __forceinline__ TileTap tile_tap(float2 o, uint32_t W, float octRes) {
    const float xl = fmaf(o.x, octRes, 0.5f), yl = fmaf(o.y, octRes, 0.5f);
    const float x0 = floorf(xl), y0 = floorf(yl);
    TileTap t;
    t.off = (uint32_t)y0 * W + (uint32_t)x0;
    t.fx = xl - x0;
    t.fy = yl - y0;
    return t;
}
__device__ __forceinline__ float4 tile_fetch(const uint2* atlas, uint32_t W, uint32_t tileOrigin, const TileTap& t) {
    const uint2* p = atlas + tileOrigin + t.off;
    const float4 t00 = half4_to_float4(__ldg(p)), t10 = half4_to_float4(__ldg(p + 1));
    const float4 t01 = half4_to_float4(__ldg(p + W)), t11 = half4_to_float4(__ldg(p + W + 1));
    const float w00 = (1.0f - t.fx) * (1.0f - t.fy), w10 = t.fx * (1.0f - t.fy), w01 = (1.0f - t.fx) * t.fy,
                w11 = t.fx * t.fy;
    return make_float4(t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11,
                       t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11,
                       t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11,
                       t00.w * w00 + t10.w * w10 + t01.w * w01 + t11.w * w11);
}

// FULL = false compiles the default receiver alone (chebyStrength 0, no dual
// detail): no depth fetch and no second fetch direction.
template <bool FULL>
__device__ float3 gather_cascade(const GatherCascade& C, const GatherArgs& A, float chebyBias, float3 cageP,
                                 float3 P, float3 Nvis, float3 Ndir, bool dual) {
    float base[3], frac[3], rm1[3];
    const float cp[3] = {cageP.x, cageP.y, cageP.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        rm1[a] = fmaxf(C.res[a] - 1.0f, 1.0f);
        const float cell = C.gridSize[a] / rm1[a];
        const float gf = (cp[a] - C.gridMin[a]) / fmaxf(cell, 1e-6f);
        base[a] = clampf(floorf(gf), 0.0f, fmaxf(C.res[a] - 2.0f, 0.0f));
        frac[a] = clampf(gf - base[a], 0.0f, 1.0f);
    }
    const float3 Nn = normalize3(Nvis);
    const TileTap tN = tile_tap(oct_encode(normalize3(Ndir)), C.atlasW, 6.0f);
    const TileTap tS = dual ? tile_tap(oct_encode(Nn), C.atlasW, 6.0f) : tN;
    const uint32_t resY = (uint32_t)C.res[1];
    const float cs = FULL ? A.chebyStrength : 0.0f;
    if (!FULL) dual = false;
    float3 acc = mk(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
#pragma unroll 2
    for (int i = 0; i < 8; ++i) {
        const int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        const float px = base[0] + float(dx), py = base[1] + float(dy), pz = base[2] + float(dz);
        const float wx = dx ? frac[0] : 1.0f - frac[0];
        const float wy = dy ? frac[1] : 1.0f - frac[1];
        const float wz = dz ? frac[2] : 1.0f - frac[2];
        const float wTri = wx * wy * wz + 1e-4f;
        const uint32_t tile = ((uint32_t)pz * resY + (uint32_t)py) * 8u * C.atlasW + (uint32_t)px * 8u;
        float w = wTri;
        if (FULL && cs != 0.0f) {
            const float3 probePos = mk(C.gridMin[0] + px / rm1[0] * C.gridSize[0],
                                       C.gridMin[1] + py / rm1[1] * C.gridSize[1],
                                       C.gridMin[2] + pz / rm1[2] * C.gridSize[2]);
            const float3 toSurf = P - probePos;
            const float dist = sqrtf(dot3(toSurf, toSurf));
            const float inv = 1.0f / fmaxf(dist, 1e-6f);
            const float4 m = tile_fetch(C.depth, C.atlasW, tile, tile_tap(oct_encode(toSurf * inv), C.atlasW, 6.0f));
            const float m1 = m.x, m2 = m.y;
            const float variance = fabsf(m2 - m1 * m1);
            const float dm = fmaxf(dist - m1 - chebyBias, 0.0f);
            const float chebyRaw = variance / fmaxf(variance + dm * dm, 1e-6f);
            const float cheby = dist <= m1 + chebyBias ? 1.0f : chebyRaw;
            const float visW = (1.0f - cs) + fmaxf(cheby * cheby * cheby, 0.05f) * cs;
            const float3 toProbe = (probePos - P) * inv;
            const float wrap = dot3(toProbe, Nn) * 0.5f + 0.5f;
            const float wrapW = (1.0f - cs) + fmaxf(wrap * wrap, 0.05f) * cs;
            w = wTri * wrapW * visW;
        }
        const float4 e4 = tile_fetch(C.atlas, C.atlasW, tile, tN);
        float3 e = mk(e4.x, e4.y, e4.z);
        if (FULL && dual) {
            const float4 eS = tile_fetch(C.atlas, C.atlasW, tile, tS);
            const float t = A.detailStrength;
            e = mk(eS.x, eS.y, eS.z) * (1.0f - t) + e * t;
        }
        acc = acc + e * w;
        wsum += w;
    }
    return acc * (1.0f / fmaxf(wsum, 1e-4f));
}

template <bool FULL>
__global__ void __launch_bounds__(256, FULL ? 3 : 4) k_gather(const GatherArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.count) return;
    const float4 p4 = __ldcs(A.position + i), n4 = __ldcs(A.stableNormal + i), d4 = __ldcs(A.detailNormal + i);
    const float3 Nvis = xyz(n4), Ndir = xyz(d4);
    const float3 reflP = xyz(p4) * A.samplePositionScale;
    const float3 P = reflP + Nvis * A.normalBias0 * A.sampleBiasScale;
    float3 E;
    if (A.cascades < 2) {
        E = gather_cascade<FULL>(A.c[0], A, A.chebyBias[0], P, P, Nvis, Ndir, A.dualDetail != 0);
    } else {
        const GatherCascade& F = A.c[1];
        const float f0 = (P.x - F.gridMin[0]) / fmaxf(F.gridSize[0], 1e-6f);
        const float f1 = (P.y - F.gridMin[1]) / fmaxf(F.gridSize[1], 1e-6f);
        const float f2 = (P.z - F.gridMin[2]) / fmaxf(F.gridSize[2], 1e-6f);
        const float fLo = fminf(fminf(f0, f1), f2);
        const float fHi = fminf(fminf(1.0f - f0, 1.0f - f1), 1.0f - f2);
        const float wIn = clampf(fminf(fLo, fHi) / fmaxf(A.borderBand, 1e-4f), 0.0f, 1.0f);
        const float wFine = wIn * clampf(float(A.cascades) - 1.0f, 0.0f, 1.0f);
        E = mk(0.0f, 0.0f, 0.0f);
        if (wFine < 1.0f) E = gather_cascade<FULL>(A.c[0], A, A.chebyBias[0], reflP, P, Nvis, Ndir, false);
        if (wFine > 0.0f) {
            const float3 Ef = gather_cascade<FULL>(A.c[1], A, A.chebyBias[1], reflP, P, Nvis, Ndir, false);
            E = E * (1.0f - wFine) + Ef * wFine;
        }
    }
    const float k = A.intensity * A.enabled;
    __stcs(A.out + i, make_float4(fmaxf(E.x, 0.0f) * k, fmaxf(E.y, 0.0f) * k, fmaxf(E.z, 0.0f) * k, 1.0f));
}


// smoothstep with the reciprocal of its (constant) edge span supplied
__device__ __forceinline__ float smoothstepf(float e0, float invSpan, float x) {
    const float t = clampf((x - e0) * invSpan, 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ float3 fast_normalize(float3 a) { return a * rsqrtf(dot3(a, a)); }

// One cascade of the combined receiver (_sampleCombinedCascadeLooped,
// gi_probes.js:662-771): the irradiance taps with the cage at the biased point
// P, and per tap with a live lobe the parallax-corrected rough / glossy fetch.
__device__ void combined_cascade(const GatherCascade& C, const GatherArgs& A, float chebyBias, float3 P, float3 reflP,
                                 float3 Nvis, float3 Ndir, float3 Rn, bool dual, float rw, float lobeMix,
                                 float3& irr, float4& refl) {
    float base[3], frac[3], cell[3];
    const float cp[3] = {P.x, P.y, P.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        cell[a] = C.gridSize[a] / fmaxf(C.res[a] - 1.0f, 1.0f);
        const float gf = (cp[a] - C.gridMin[a]) / fmaxf(cell[a], 1e-6f);
        base[a] = clampf(floorf(gf), 0.0f, fmaxf(C.res[a] - 2.0f, 0.0f));
        frac[a] = clampf(gf - base[a], 0.0f, 1.0f);
    }
    const float3 Nn = normalize3(Nvis);
    const TileTap tN = tile_tap(oct_encode(normalize3(Ndir)), C.atlasW, 6.0f);
    const TileTap tS = dual ? tile_tap(oct_encode(Nn), C.atlasW, 6.0f) : tN;
    const TileTap tR = tile_tap(oct_encode(Rn), C.atlasW, 6.0f);
    const uint32_t resX = (uint32_t)C.res[0], resY = (uint32_t)C.res[1], resXY = resX * resY;
    const float cs = A.chebyStrength;
    const bool glossyOn = C.glossy != nullptr;
    const bool wantsRough = lobeMix > 0.0f, wantsGlossy = glossyOn && lobeMix < 1.0f;
    const bool wantsTap = rw > 0.0f && (wantsRough || wantsGlossy);
    float3 acc = mk(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f, roughW = 0.0f, glossyW = 0.0f;
    float4 roughAcc = make_float4(0.f, 0.f, 0.f, 0.f), glossyAcc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < 8; ++i) {
        const int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        const float px = base[0] + float(dx), py = base[1] + float(dy), pz = base[2] + float(dz);
        const float wx = dx ? frac[0] : 1.0f - frac[0];
        const float wy = dy ? frac[1] : 1.0f - frac[1];
        const float wz = dz ? frac[2] : 1.0f - frac[2];
        const float wTri = wx * wy * wz + 1e-4f;
        const uint32_t tile = ((uint32_t)pz * resY + (uint32_t)py) * 8u * C.atlasW + (uint32_t)px * 8u;
        // the probe at grid index (px, py, pz): gridMin + p * cell (within an ulp of
        // the reference's gridMin + p / (res - 1) * gridSize)
        const float3 probePos = mk(fmaf(px, cell[0], C.gridMin[0]), fmaf(py, cell[1], C.gridMin[1]),
                                   fmaf(pz, cell[2], C.gridMin[2]));
        float w = wTri;
        if (cs != 0.0f) {
            const float3 toSurf = P - probePos;
            const float dist = sqrtf(dot3(toSurf, toSurf));
            const float inv = 1.0f / fmaxf(dist, 1e-6f);
            const float4 m = tile_fetch(C.depth, C.atlasW, tile, tile_tap(oct_encode(toSurf * inv), C.atlasW, 6.0f));
            const float variance = fabsf(m.y - m.x * m.x);
            const float dm = fmaxf(dist - m.x - chebyBias, 0.0f);
            const float chebyRaw = variance / fmaxf(variance + dm * dm, 1e-6f);
            const float cheby = dist <= m.x + chebyBias ? 1.0f : chebyRaw;
            const float visW = (1.0f - cs) + fmaxf(cheby * cheby * cheby, 0.05f) * cs;
            const float wrap = dot3((probePos - P) * inv, Nn) * 0.5f + 0.5f;
            const float wrapW = (1.0f - cs) + fmaxf(wrap * wrap, 0.05f) * cs;
            w = wTri * wrapW * visW;
        }
        const float4 e4 = tile_fetch(C.atlas, C.atlasW, tile, tN);
        float3 e = mk(e4.x, e4.y, e4.z);
        if (dual) {
            const float4 eS = tile_fetch(C.atlas, C.atlasW, tile, tS);
            e = mk(eS.x, eS.y, eS.z) * (1.0f - A.detailStrength) + e * A.detailStrength;
        }
        acc = acc + e * w;
        wsum += w;
        if (!wantsTap) continue;
        // the reflection ray against the sphere of the probe's mean depth toward R
        const float4 dR = tile_fetch(C.depth, C.atlasW, tile, tR);
        const float radius = fmaxf(dR.x, 1e-4f), radius2 = radius * radius;
        const float3 q = reflP - probePos;
        const float q2 = dot3(q, q), qDotR = dot3(q, Rn);
        // radius^2 - q^2 + (q.R)^2 with |R| = 1 is radius^2 - |q x R|^2: the cross
        // product keeps the two nearly equal squares from cancelling in FP32
        const float3 qxR = cross3(q, Rn);
        const float disc = radius2 - dot3(qxR, qxR);
        const float sqrtDisc = sqrtf(fmaxf(disc, 0.0f));
        const float nearT = -qDotR - sqrtDisc, farT = -qDotR + sqrtDisc;
        const float rayT = nearT > 1e-4f ? nearT : farT;
        const float invR2 = 1.0f / fmaxf(radius2, 1e-4f);
        const float relVar = fmaxf(dR.y - radius2, 0.0f) * invR2;
        const float stableDepth = 1.0f - smoothstepf(0.02f, 1.0f / 0.18f, relVar);
        const float validHit = (disc > 1e-6f && rayT > 1e-4f) ? 1.0f : 0.0f;
        const float insideWeight = smoothstepf(0.0f, 1.0f / 0.12f, (radius2 - q2) * invR2);
        const float pw = stableDepth * validHit * insideWeight;
        const float3 corrected = fast_normalize(q + Rn * fmaxf(rayT, 0.0f));
        const float2 oSR = oct_encode(fast_normalize(Rn * (1.0f - pw) + corrected * pw));
        const float probeW = w * w;
        if (wantsGlossy) {
            // the probe's glossy tile: the index and its row and column are exact integers
            const uint32_t probeIndex = (uint32_t)px + (uint32_t)py * resX + (uint32_t)pz * resXY;
            const uint32_t gtile = (probeIndex / C.glossyTilesX) * C.glossyTile * C.glossyW +
                                   (probeIndex % C.glossyTilesX) * C.glossyTile;
            const float4 gl = tile_fetch(C.glossy, C.glossyW, gtile, tile_tap(oSR, C.glossyW, float(C.glossyOct)));
            const float gw = probeW * (0.2f * (1.0f - pw) + pw);
            glossyAcc = make_float4(glossyAcc.x + gl.x * gw, glossyAcc.y + gl.y * gw, glossyAcc.z + gl.z * gw,
                                    glossyAcc.w + gl.w * gw);
            glossyW += gw;
        }
        if (wantsRough) {
            const float4 br = tile_fetch(C.rough, C.atlasW, tile, tile_tap(oSR, C.atlasW, 6.0f));
            roughAcc = make_float4(roughAcc.x + br.x * probeW, roughAcc.y + br.y * probeW, roughAcc.z + br.z * probeW,
                                   roughAcc.w + br.w * probeW);
            roughW += probeW;
        }
    }
    irr = acc * (1.0f / fmaxf(wsum, 1e-4f));
    const float ri = 1.0f / fmaxf(roughW, 1e-4f);
    refl = make_float4(roughAcc.x * ri, roughAcc.y * ri, roughAcc.z * ri, roughAcc.w * ri);
    if (glossyOn) {
        const float gi = 1.0f / fmaxf(glossyW, 1e-4f);
        refl = make_float4(glossyAcc.x * gi * (1.0f - lobeMix) + refl.x * lobeMix,
                           glossyAcc.y * gi * (1.0f - lobeMix) + refl.y * lobeMix,
                           glossyAcc.z * gi * (1.0f - lobeMix) + refl.z * lobeMix,
                           glossyAcc.w * gi * (1.0f - lobeMix) + refl.w * lobeMix);
    }
}

__global__ void __launch_bounds__(256, 3) k_gather_combined(const GatherArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.count) return;
    const float4 p4 = __ldcs(A.position + i), n4 = __ldcs(A.stableNormal + i), d4 = __ldcs(A.detailNormal + i);
    const float4 r4 = __ldcs(A.reflection + i);
    const float3 Nvis = xyz(n4), Ndir = xyz(d4), Rn = normalize3(xyz(r4));
    const float roughness = r4.w;
    const float3 reflP = xyz(p4) * A.samplePositionScale;
    const float3 P = reflP + Nvis * A.normalBias0 * A.sampleBiasScale;
    const float part = roughness <= A.roughnessLimit ? 1.0f : 0.0f;
    const float rw = clampf(A.reflectionIntensity * A.enabled * part, 0.0f, 1.0f);
    const float lobeMix = A.c[0].glossy ? smoothstepf(0.22f, 1.0f / 0.36f, roughness) : 1.0f;
    float3 E;
    float4 S;
    if (A.cascades < 2) {
        combined_cascade(A.c[0], A, A.chebyBias[0], P, reflP, Nvis, Ndir, Rn, A.dualDetail != 0, rw, lobeMix, E, S);
    } else {
        // cascade ownership at the surface position (gi_probes.js:787-792)
        const GatherCascade& F = A.c[1];
        const float f0 = (reflP.x - F.gridMin[0]) / fmaxf(F.gridSize[0], 1e-6f);
        const float f1 = (reflP.y - F.gridMin[1]) / fmaxf(F.gridSize[1], 1e-6f);
        const float f2 = (reflP.z - F.gridMin[2]) / fmaxf(F.gridSize[2], 1e-6f);
        const float fLo = fminf(fminf(f0, f1), f2);
        const float fHi = fminf(fminf(1.0f - f0, 1.0f - f1), 1.0f - f2);
        const float wIn = clampf(fminf(fLo, fHi) / fmaxf(A.borderBand, 1e-4f), 0.0f, 1.0f);
        const float wFine = wIn * clampf(float(A.cascades) - 1.0f, 0.0f, 1.0f);
        E = mk(0.0f, 0.0f, 0.0f);
        S = make_float4(0.f, 0.f, 0.f, 0.f);
        if (wFine < 1.0f) combined_cascade(A.c[0], A, A.chebyBias[0], P, reflP, Nvis, Ndir, Rn, false, rw, lobeMix, E, S);
        if (wFine > 0.0f) {
            float3 Ef;
            float4 Sf;
            combined_cascade(A.c[1], A, A.chebyBias[1], P, reflP, Nvis, Ndir, Rn, false, rw, lobeMix, Ef, Sf);
            E = E * (1.0f - wFine) + Ef * wFine;
            S = make_float4(S.x * (1.0f - wFine) + Sf.x * wFine, S.y * (1.0f - wFine) + Sf.y * wFine,
                            S.z * (1.0f - wFine) + Sf.z * wFine, S.w * (1.0f - wFine) + Sf.w * wFine);
        }
    }
    const float k = A.intensity * A.enabled;
    __stcs(A.out + i, make_float4(fmaxf(E.x, 0.0f) * k, fmaxf(E.y, 0.0f) * k, fmaxf(E.z, 0.0f) * k, 1.0f));
    const float4 o = rw > 0.0f ? make_float4(fmaxf(S.x, 0.0f) * rw, fmaxf(S.y, 0.0f) * rw, fmaxf(S.z, 0.0f) * rw,
                                             clampf(fmaxf(S.w, 0.0f), 0.0f, 1.0f) * rw)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
    __stcs(A.outReflection + i, o);
}

}  // namespace

cudaError_t launch_gather_combined(const GatherArgs& A, cudaStream_t st) {
    if (A.count == 0) return cudaSuccess;
    k_gather_combined<<<(A.count + 255) / 256, 256, 0, st>>>(A);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs& A, cudaStream_t st) {
    if (A.count == 0) return cudaSuccess;
    const bool full = A.cascades > 1 || A.chebyStrength != 0.0f || A.dualDetail;
    if (full) k_gather<true><<<(A.count + 255) / 256, 256, 0, st>>>(A);
    else k_gather<false><<<(A.count + 255) / 256, 256, 0, st>>>(A);
    note_launch();
    return cudaGetLastError();
}

}  // namespace sb
