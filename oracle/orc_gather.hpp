// orc_gather.hpp — restatement of the receiver gather, the consumer of the
// atlases: GiProbeNode.setup's sample point (gi_probes.js:884-885, 927-928),
// sampleIrradiance (816-850), _sampleCascade (583-614), _sampleCascadeLooped
// (625-657), _tapEW (530-579), _probePos (483-486) and _tileUV (488-497).
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
//
// Classification is inert (classifyStrength 0, gi_probes.js:358): the state
// atlas's relocation is scaled to zero and the state weight is mix(1, s, 0) = 1,
// so no state atlas is read. With chebyStrength 0 (the default, 355) the
// visibility and wrap weights are mix(1, x, 0) = 1 for any finite x; the depth
// atlas is then not read either.
// The looped (two-cascade) gather chooses its probe cage at the unbiased
// surface position, as its comment states (628-631); the code names
// `reflectionP` there, which is not in that function's scope.
#pragma once
#include "orc_probes.hpp"

namespace orc {

struct GatherParams {
    double normalBias[2], chebyBias[2];
    double chebyStrength, detailStrength, intensity, enabled;
    double samplePositionScale, sampleBiasScale, borderBand;
    double cascades, dualDetail;
    double reflectionIntensity, roughnessLimit;  // setReflectionIntensity / setRoughnessLimit (gi_probes.js:412-419)
};

struct GatherCascade {
    const Grid* g = nullptr;
    const uint16_t* atlas = nullptr;
    const uint16_t* depth = nullptr;
    // reflection lobes (the combined receiver): rough atlas in the irradiance
    // layout; glossy atlas of glossyTile-texel tiles, glossyTilesX to a row
    const uint16_t* rough = nullptr;
    const uint16_t* glossy = nullptr;
    uint32_t glossyOct = 0, glossyTile = 0, glossyTilesX = 1, glossyW = 1, glossyH = 1;
};

template <class R> inline V3<R> tile_uv(const Grid& g, R col, R row, R ou, R ov) {
    R ox = col * R(TILE) + R(BORDER) + ou * R(OCT_RES);
    R oy = row * R(TILE) + R(BORDER) + ov * R(OCT_RES);
    return V3<R>(ox / R(g.atlasW()), oy / R(g.atlasH()), R(0));
}

// Distance of x to the nearest integer (the cage-selection discontinuity).
inline double frac_dist(double x) { return std::fabs(x - std::floor(x + 0.5)); }

// One cascade's 8-tap gather. `cageP` picks the cage, `P` is the biased point.
// `near` records how close the evaluation came to a discontinuity (cage floor
// in cell units; Chebyshev select relative to the distance).
template <class R>
V3<R> gather_cascade(const GatherCascade& C, int c, const GatherParams& prm, V3<R> cageP, V3<R> P, V3<R> Nvis,
                     V3<R> Ndir, bool dual, double& near) {
    const Grid& g = *C.g;
    R resv[3] = {R(g.res[0]), R(g.res[1]), R(g.res[2])};
    R gmin[3] = {R(g.gridMin[0]), R(g.gridMin[1]), R(g.gridMin[2])};
    R gsz[3] = {R(g.gridSize[0]), R(g.gridSize[1]), R(g.gridSize[2])};
    R cp[3] = {cageP.x, cageP.y, cageP.z};
    R base[3], frac[3];
    for (int a = 0; a < 3; ++a) {
        R cell = gsz[a] / std::max(resv[a] - R(1), R(1));
        R gf = (cp[a] - gmin[a]) / std::max(cell, R(1e-6));
        base[a] = clampv(std::floor(gf), R(0), std::max(resv[a] - R(2), R(0)));
        frac[a] = clampv(gf - base[a], R(0), R(1));
        near = std::min(near, frac_dist((double)gf));
    }
    V3<R> Nn = normalize(Nvis);
    R onu, onv, osu = 0, osv = 0;
    oct_encode(normalize(Ndir), onu, onv);
    if (dual) oct_encode(Nn, osu, osv);
    const R cs = R(prm.chebyStrength);
    V3<R> acc;
    R wsum = 0;
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        R px = base[0] + R(dx), py = base[1] + R(dy), pz = base[2] + R(dz);
        R wx = dx ? frac[0] : R(1) - frac[0];
        R wy = dy ? frac[1] : R(1) - frac[1];
        R wz = dz ? frac[2] : R(1) - frac[2];
        R wTri = wx * wy * wz + R(1e-4);
        R col = px, row = pz * resv[1] + py;
        R w = wTri;
        if (cs != R(0)) {
            V3<R> probePos(gmin[0] + px / std::max(resv[0] - R(1), R(1)) * gsz[0],
                           gmin[1] + py / std::max(resv[1] - R(1), R(1)) * gsz[1],
                           gmin[2] + pz / std::max(resv[2] - R(1), R(1)) * gsz[2]);
            V3<R> toSurf = P - probePos;
            R dist = length(toSurf);
            R du, dv;
            oct_encode(toSurf * (R(1) / std::max(dist, R(1e-6))), du, dv);
            V3<R> uv = tile_uv<R>(g, col, row, du, dv);
            V3<R> m = bilinear_rgb<R>(C.depth, g.atlasW(), g.atlasH(), uv.x, uv.y);
            R m1 = m.x, m2 = m.y;
            R variance = std::fabs(m2 - m1 * m1);
            R db = R(prm.chebyBias[c]);
            R dm = std::max(dist - m1 - db, R(0));
            R chebyRaw = variance / std::max(variance + dm * dm, R(1e-6));
            R cheby = dist <= m1 + db ? R(1) : chebyRaw;
            near = std::min(near, std::fabs((double)(dist - (m1 + db))) / std::max(1.0, (double)dist));
            R visW = R(1) * (R(1) - cs) + std::max(cheby * cheby * cheby, R(0.05)) * cs;
            V3<R> dirToProbe = (probePos - P) * (R(1) / std::max(dist, R(1e-6)));
            R wrap = dot(dirToProbe, Nn) * R(0.5) + R(0.5);
            R wrapW = R(1) * (R(1) - cs) + std::max(wrap * wrap, R(0.05)) * cs;
            w = wTri * wrapW * visW;
        }
        V3<R> uvD = tile_uv<R>(g, col, row, onu, onv);
        V3<R> e = bilinear_rgb<R>(C.atlas, g.atlasW(), g.atlasH(), uvD.x, uvD.y);
        if (dual) {
            V3<R> uvS = tile_uv<R>(g, col, row, osu, osv);
            V3<R> eS = bilinear_rgb<R>(C.atlas, g.atlasW(), g.atlasH(), uvS.x, uvS.y);
            R t = R(prm.detailStrength);
            e = eS * (R(1) - t) + e * t;
        }
        acc = acc + e * w;
        wsum += w;
    }
    return acc * (R(1) / std::max(wsum, R(1e-4)));
}

// The receiver's irradiance at one surface point: E = max(sample, 0) *
// intensity * enabled (gi_probes.js:927-928).
template <class R>
V3<R> gather_point(const GatherCascade C[2], const GatherParams& prm, V3<R> pos, V3<R> Nvis, V3<R> Ndir, double& near) {
    V3<R> reflP = pos * R(prm.samplePositionScale);
    V3<R> P = reflP + Nvis * R(prm.normalBias[0]) * R(prm.sampleBiasScale);
    V3<R> E;
    const bool useFine = prm.cascades >= 2 && C[1].g && C[1].atlas;
    if (!useFine) {
        E = gather_cascade<R>(C[0], 0, prm, P, P, Nvis, Ndir, prm.dualDetail != 0, near);
    } else {
        const Grid& g1 = *C[1].g;
        R f[3];
        for (int a = 0; a < 3; ++a)
            f[a] = ((&P.x)[a] - R(g1.gridMin[a])) / std::max(R(g1.gridSize[a]), R(1e-6));
        R fLo = std::min(std::min(f[0], f[1]), f[2]);
        R fHi = std::min(std::min(R(1) - f[0], R(1) - f[1]), R(1) - f[2]);
        R edge = std::min(fLo, fHi);
        R wIn = clampv(edge / std::max(R(prm.borderBand), R(1e-4)), R(0), R(1));
        R gate = clampv(R(prm.cascades) - R(1), R(0), R(1));
        R wFine = wIn * gate;
        if (wFine < R(1)) E = gather_cascade<R>(C[0], 0, prm, reflP, P, Nvis, Ndir, false, near);
        if (wFine > R(0)) {
            V3<R> Ef = gather_cascade<R>(C[1], 1, prm, reflP, P, Nvis, Ndir, false, near);
            E = E * (R(1) - wFine) + Ef * wFine;
        }
    }
    R k = R(prm.intensity) * R(prm.enabled);
    return V3<R>(std::max(E.x, R(0)) * k, std::max(E.y, R(0)) * k, std::max(E.z, R(0)) * k);
}

// ---------------------------------------------------------------------------
// The combined receiver: diffuse irradiance and the local reflection of the
// rough / glossy lobes in one pass (GiProbeNode._sampleCombinedCascadeLooped,
// gi_probes.js:658-771; sampleIrradianceAndRough 773-806; the reflection branch
// of setup 893-925; _glossyTileUV 498-507).

template <class R, class T> inline void bilinear_rgba(const T* atlas, uint32_t W, uint32_t H, R u, R v, R out[4]) {
    R x = u * R(W) - R(0.5), y = v * R(H) - R(0.5);
    R fx0 = std::floor(x), fy0 = std::floor(y);
    R fx = x - fx0, fy = y - fy0;
    long x0 = (long)fx0, y0 = (long)fy0;
    auto cl = [](long a, long n) { return a < 0 ? 0 : (a >= n ? n - 1 : a); };
    long xs[2] = {cl(x0, W), cl(x0 + 1, W)}, ys[2] = {cl(y0, H), cl(y0 + 1, H)};
    R wxs[2] = {R(1) - fx, fx}, wys[2] = {R(1) - fy, fy};
    for (int c = 0; c < 4; ++c) out[c] = R(0);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            const T* t = atlas + ((size_t)ys[j] * W + xs[i]) * 4;
            R w = wxs[i] * wys[j];
            for (int c = 0; c < 4; ++c) out[c] += R(texel_value(t[c])) * w;
        }
}

template <class R> inline R smoothstep_(R e0, R e1, R x) {
    R t = clampv((x - e0) / (e1 - e0), R(0), R(1));
    return t * t * (R(3) - R(2) * t);
}

constexpr double ROUGH_LOBE_MIX_START = 0.22, ROUGH_LOBE_MIX_END = 0.58;        // gi_probes.js:83-84
constexpr double ROUGH_PARALLAX_VAR_START = 0.02, ROUGH_PARALLAX_VAR_END = 0.20;  // 88-89
constexpr double ROUGH_PARALLAX_INSIDE_FADE = 0.12;                              // 90

// One cascade of the combined receiver: the irradiance taps of the looped
// gather (cage at the biased point P) and, per tap with a live lobe, the
// parallax-corrected lookup of the rough and glossy atlases. irr: 3, refl: 4.
template <class R>
void combined_cascade(const GatherCascade& C, int c, const GatherParams& prm, V3<R> P, V3<R> reflP, V3<R> Nvis,
                      V3<R> Ndir, V3<R> Rn, bool dual, R reflectionWeight, R roughLobeMix, double& near, V3<R>& irr,
                      R refl[4]) {
    const Grid& g = *C.g;
    const bool glossyOn = C.glossy != nullptr;
    R resv[3] = {R(g.res[0]), R(g.res[1]), R(g.res[2])};
    R gmin[3] = {R(g.gridMin[0]), R(g.gridMin[1]), R(g.gridMin[2])};
    R gsz[3] = {R(g.gridSize[0]), R(g.gridSize[1]), R(g.gridSize[2])};
    R pp[3] = {P.x, P.y, P.z};
    R base[3], frac[3];
    for (int a = 0; a < 3; ++a) {
        R cell = gsz[a] / std::max(resv[a] - R(1), R(1));
        R gf = (pp[a] - gmin[a]) / std::max(cell, R(1e-6));
        base[a] = clampv(std::floor(gf), R(0), std::max(resv[a] - R(2), R(0)));
        frac[a] = clampv(gf - base[a], R(0), R(1));
        near = std::min(near, frac_dist((double)gf));
    }
    V3<R> Nn = normalize(Nvis);
    R onu, onv, osu = 0, osv = 0, oru, orv;
    oct_encode(normalize(Ndir), onu, onv);
    if (dual) oct_encode(Nn, osu, osv);
    oct_encode(Rn, oru, orv);
    const R cs = R(prm.chebyStrength);
    V3<R> acc;
    R wsum = 0, roughAcc[4] = {0, 0, 0, 0}, glossyAcc[4] = {0, 0, 0, 0}, roughW = 0, glossyW = 0;
    const bool wantsRough = roughLobeMix > R(0);
    const bool wantsGlossy = glossyOn && roughLobeMix < R(1);
    const bool wantsTap = reflectionWeight > R(0) && (wantsRough || wantsGlossy);
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        R px = base[0] + R(dx), py = base[1] + R(dy), pz = base[2] + R(dz);
        R wx = dx ? frac[0] : R(1) - frac[0];
        R wy = dy ? frac[1] : R(1) - frac[1];
        R wz = dz ? frac[2] : R(1) - frac[2];
        R wTri = wx * wy * wz + R(1e-4);
        R col = px, row = pz * resv[1] + py;
        V3<R> probePos(gmin[0] + px / std::max(resv[0] - R(1), R(1)) * gsz[0],
                       gmin[1] + py / std::max(resv[1] - R(1), R(1)) * gsz[1],
                       gmin[2] + pz / std::max(resv[2] - R(1), R(1)) * gsz[2]);
        R w = wTri;
        if (cs != R(0)) {
            V3<R> toSurf = P - probePos;
            R dist = length(toSurf);
            R du, dv;
            oct_encode(toSurf * (R(1) / std::max(dist, R(1e-6))), du, dv);
            V3<R> uv = tile_uv<R>(g, col, row, du, dv);
            V3<R> m = bilinear_rgb<R>(C.depth, g.atlasW(), g.atlasH(), uv.x, uv.y);
            R variance = std::fabs(m.y - m.x * m.x);
            R db = R(prm.chebyBias[c]);
            R dm = std::max(dist - m.x - db, R(0));
            R chebyRaw = variance / std::max(variance + dm * dm, R(1e-6));
            R cheby = dist <= m.x + db ? R(1) : chebyRaw;
            near = std::min(near, std::fabs((double)(dist - (m.x + db))) / std::max(1.0, (double)dist));
            R visW = R(1) * (R(1) - cs) + std::max(cheby * cheby * cheby, R(0.05)) * cs;
            V3<R> dirToProbe = (probePos - P) * (R(1) / std::max(dist, R(1e-6)));
            R wrap = dot(dirToProbe, Nn) * R(0.5) + R(0.5);
            R wrapW = R(1) * (R(1) - cs) + std::max(wrap * wrap, R(0.05)) * cs;
            w = wTri * wrapW * visW;
        }
        V3<R> uvD = tile_uv<R>(g, col, row, onu, onv);
        V3<R> e = bilinear_rgb<R>(C.atlas, g.atlasW(), g.atlasH(), uvD.x, uvD.y);
        if (dual) {
            V3<R> uvS = tile_uv<R>(g, col, row, osu, osv);
            V3<R> eS = bilinear_rgb<R>(C.atlas, g.atlasW(), g.atlasH(), uvS.x, uvS.y);
            R t = R(prm.detailStrength);
            e = eS * (R(1) - t) + e * t;
        }
        acc = acc + e * w;
        wsum += w;
        if (!wantsTap) continue;
        // parallax: the reflection ray against the sphere of the probe's mean depth toward R
        V3<R> uvR = tile_uv<R>(g, col, row, oru, orv);
        V3<R> depthR = bilinear_rgb<R>(C.depth, g.atlasW(), g.atlasH(), uvR.x, uvR.y);
        R radius = std::max(depthR.x, R(1e-4)), radius2 = radius * radius;
        V3<R> q = reflP - probePos;
        R q2 = dot(q, q), qDotR = dot(q, Rn);
        R disc = radius2 - q2 + qDotR * qDotR;
        R sqrtDisc = std::sqrt(std::max(disc, R(0)));
        R nearT = -qDotR - sqrtDisc, farT = -qDotR + sqrtDisc;
        R rayT = nearT > R(1e-4) ? nearT : farT;
        near = std::min(near, std::fabs((double)(nearT - R(1e-4))) / std::max(1.0, std::fabs((double)nearT)));
        near = std::min(near, std::fabs((double)(farT - R(1e-4))) / std::max(1.0, std::fabs((double)farT)));
        near = std::min(near, std::fabs((double)(disc - R(1e-6))) / std::max(1.0, (double)radius2));
        R relVar = std::max(depthR.y - radius2, R(0)) / std::max(radius2, R(1e-4));
        R stableDepth = R(1) - smoothstep_(R(ROUGH_PARALLAX_VAR_START), R(ROUGH_PARALLAX_VAR_END), relVar);
        R validHit = (disc > R(1e-6) && rayT > R(1e-4)) ? R(1) : R(0);
        R insideRatio = (radius2 - q2) / std::max(radius2, R(1e-4));
        R insideWeight = smoothstep_(R(0), R(ROUGH_PARALLAX_INSIDE_FADE), insideRatio);
        R parallaxWeight = stableDepth * validHit * insideWeight;
        V3<R> correctedR = normalize(q + Rn * std::max(rayT, R(0)));
        V3<R> sampleR = normalize(Rn * (R(1) - parallaxWeight) + correctedR * parallaxWeight);
        R osr, osv2;
        oct_encode(sampleR, osr, osv2);
        R probeW = w * w;
        if (wantsGlossy) {
            R probeIndex = px + py * resv[0] + pz * (resv[0] * resv[1]);
            R tx = R(C.glossyTilesX);
            R gcol = std::fmod(probeIndex, tx), grow = std::floor(probeIndex / tx);
            R ox = gcol * R(C.glossyTile) + R(BORDER) + osr * R(C.glossyOct);
            R oy = grow * R(C.glossyTile) + R(BORDER) + osv2 * R(C.glossyOct);
            R gl[4];
            bilinear_rgba<R>(C.glossy, C.glossyW, C.glossyH, ox / R(C.glossyW), oy / R(C.glossyH), gl);
            R conf = R(0.2) * (R(1) - parallaxWeight) + R(1) * parallaxWeight;
            R gw = probeW * conf;
            for (int k = 0; k < 4; ++k) glossyAcc[k] += gl[k] * gw;
            glossyW += gw;
        }
        if (wantsRough) {
            V3<R> uvB = tile_uv<R>(g, col, row, osr, osv2);
            R br[4];
            bilinear_rgba<R>(C.rough, g.atlasW(), g.atlasH(), uvB.x, uvB.y, br);
            for (int k = 0; k < 4; ++k) roughAcc[k] += br[k] * probeW;
            roughW += probeW;
        }
    }
    irr = acc * (R(1) / std::max(wsum, R(1e-4)));
    for (int k = 0; k < 4; ++k) {
        R rr = roughAcc[k] / std::max(roughW, R(1e-4));
        refl[k] = glossyOn ? (glossyAcc[k] / std::max(glossyW, R(1e-4))) * (R(1) - roughLobeMix) + rr * roughLobeMix : rr;
    }
}

// The combined receiver at one surface point: irradiance E = max(E, 0) *
// intensity * enabled, and the reflection layer (rgb premultiplied by its
// weight, coverage x weight) that setup composites over the prior radiance:
// radiance * (1 - out.w) + out.rgb. rdir4 = (reflection direction, roughness).
template <class R>
void combined_point(const GatherCascade C[2], const GatherParams& prm, V3<R> pos, V3<R> Nvis, V3<R> Ndir,
                    V3<R> Rdir, R roughness, double& near, V3<R>& E, R out[4]) {
    V3<R> reflP = pos * R(prm.samplePositionScale);
    V3<R> P = reflP + Nvis * R(prm.normalBias[0]) * R(prm.sampleBiasScale);
    V3<R> Rn = normalize(Rdir);
    R part = roughness <= R(prm.roughnessLimit) ? R(1) : R(0);
    near = std::min(near, std::fabs((double)(roughness - R(prm.roughnessLimit))));
    R rw = clampv(R(prm.reflectionIntensity) * R(prm.enabled) * part, R(0), R(1));
    R mixv_ = C[0].glossy ? smoothstep_(R(ROUGH_LOBE_MIX_START), R(ROUGH_LOBE_MIX_END), roughness) : R(1);
    V3<R> irr;
    R S[4] = {0, 0, 0, 0};
    const bool useFine = prm.cascades >= 2 && C[1].g && C[1].atlas;
    if (!useFine) {
        combined_cascade<R>(C[0], 0, prm, P, reflP, Nvis, Ndir, Rn, prm.dualDetail != 0, rw, mixv_, near, irr, S);
    } else {
        const Grid& g1 = *C[1].g;
        R f[3];
        for (int a = 0; a < 3; ++a)
            f[a] = ((&reflP.x)[a] - R(g1.gridMin[a])) / std::max(R(g1.gridSize[a]), R(1e-6));
        R fLo = std::min(std::min(f[0], f[1]), f[2]);
        R fHi = std::min(std::min(R(1) - f[0], R(1) - f[1]), R(1) - f[2]);
        R wIn = clampv(std::min(fLo, fHi) / std::max(R(prm.borderBand), R(1e-4)), R(0), R(1));
        R wFine = wIn * clampv(R(prm.cascades) - R(1), R(0), R(1));
        if (wFine < R(1)) combined_cascade<R>(C[0], 0, prm, P, reflP, Nvis, Ndir, Rn, false, rw, mixv_, near, irr, S);
        if (wFine > R(0)) {
            V3<R> irrF;
            R SF[4];
            combined_cascade<R>(C[1], 1, prm, P, reflP, Nvis, Ndir, Rn, false, rw, mixv_, near, irrF, SF);
            irr = irr * (R(1) - wFine) + irrF * wFine;
            for (int k = 0; k < 4; ++k) S[k] = S[k] * (R(1) - wFine) + SF[k] * wFine;
        }
    }
    R k = R(prm.intensity) * R(prm.enabled);
    E = V3<R>(std::max(irr.x, R(0)) * k, std::max(irr.y, R(0)) * k, std::max(irr.z, R(0)) * k);
    if (rw > R(0)) {
        for (int c = 0; c < 3; ++c) out[c] = std::max(S[c], R(0)) * rw;
        out[3] = clampv(std::max(S[3], R(0)), R(0), R(1)) * rw;
    } else {
        for (int c = 0; c < 4; ++c) out[c] = R(0);
    }
}

}  // namespace orc
