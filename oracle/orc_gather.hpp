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
};

struct GatherCascade {
    const Grid* g = nullptr;
    const uint16_t* atlas = nullptr;
    const uint16_t* depth = nullptr;
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

}  // namespace orc
