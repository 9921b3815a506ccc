// orc_probes.hpp — restatement of the probe-field kernels of gi_probes.js:
// traceKernel (1977-2214, clustered NEE 2064-2127), lightGridKernel
// (1888-1938), sampleAtlas (1941-1974), blendKernel (2317-2532) and
// uploadKernel (2737-2846).
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
#pragma once
#include "orc_traverse.hpp"

namespace orc {

// Shared compute uniforms U, gi_probes.js:1198-1255 (same field order as the
// library's sb_params, stored in double).
struct Params {
    double frameJitter, emitterVisSeed;
    double hysteresis, hysteresisExponent;
    double depthSharpness, radianceClamp, classifyStrength;
    double filterStrength, filterSmooth;
    double tempChangeSigma1, tempChangeHDrop, tempClampSigma;
    double nirGate, nirGain;
    double skyIntensity;
    double skySH[27];
    double debugTraceBiasScale, debugRayEpsScale, debugDirectScale, debugEmissiveScale;
    double debugAlbedoScale, debugBounceScale, debugCosinePower;
    double debugTempNoiseHBoost, debugTempChangeSigma0, debugTempMinChangeH;
    double debugTempVarEps, debugTempVarRel, debugDepthHistoryScale;
    double debugFilterKScale, debugFilterRelScale, debugFilterEpsScale;
    double reflectionSkyFallback, skyConfigured;  // gi_probes.js:1234, 1238, 1316-1324
};

struct Lights {
    const float* data = nullptr;  // arena: 64 x 17 records (+ C0 cell lists when clustered)
    uint32_t dataLen = 0;
    uint32_t lightCount = 0;
    int clustered = 0;
    uint32_t emitterBase = 0, emitterCount = 0;  // the giEmitter records (type 3), after the analytic ones
};

constexpr uint32_t GI_EMITTER_INJECT_CAP = 16;      // gi_probes.js:133
constexpr double GI_EMITTER_VIS_RETENTION = 0.8;    // gi_probes.js:134
constexpr double ROUGH_UNSHADED_T_BIAS = 2.0;        // gi_probes.js:94

// One ray's outputs. hitT = -1 on a miss (gi_probes.js:1987, 2209-2213).
template <class R> struct RayOut {
    R rgb[3];
    R hitT;
    int tri, inst;
    R secondT;            // second-nearest accepted candidate (near-tie rule)
    uint64_t tested;      // NEE lights whose shadow ray was traced
    uint64_t blocked;     // ... and found blocked
    int facing = -1;      // hit: 1 when the geometric normal faced the ray (front side)
};

// Replay input: the GPU's own hit decision and shadow bits for one ray.
struct Replay {
    const int32_t* tri;      // per ray, -1 = miss
    const int32_t* inst;
    const uint64_t* blocked; // per ray shadow bits (light index)
};

// lightGridKernel, gi_probes.js:1893-1937: C0 cell lists after the 64x17 records.
template <class R> void light_grid(const Grid& g0, const float* lightsIn, uint32_t lightCount, float* out) {
    uint32_t cellsX = g0.res[0] - 1, cellsY = g0.res[1] - 1, cellsZ = g0.res[2] - 1;
    uint32_t cells = std::max(1u, cellsX) * std::max(1u, cellsY) * std::max(1u, cellsZ);
    for (uint32_t c = 0; c < cells; ++c) {
        uint32_t ix = c % cellsX, iy = (c / cellsX) % cellsY, iz = c / (cellsX * cellsY);
        V3<R> cellSize(R(g0.gridSize[0]) / R(cellsX), R(g0.gridSize[1]) / R(cellsY), R(g0.gridSize[2]) / R(cellsZ));
        V3<R> cmin = V3<R>(R(g0.gridMin[0]), R(g0.gridMin[1]), R(g0.gridMin[2])) + mulv(V3<R>(R(ix), R(iy), R(iz)), cellSize);
        V3<R> cmax = cmin + cellSize;
        size_t listBase = (size_t)MAX_LIGHTS * LIGHT_STRIDE + (size_t)c * LIGHT_CELL_STRIDE;
        uint32_t count = 0;
        for (uint32_t li = 0; li < lightCount; ++li) {
            const float* L = lightsIn + (size_t)li * LIGHT_STRIDE;
            R ltype = R(L[0]);
            V3<R> lpos{R(L[1]), R(L[2]), R(L[3])};
            R lrange = R(L[10]);
            R dx = std::max(std::max(cmin.x - lpos.x, R(0)), lpos.x - cmax.x);
            R dy = std::max(std::max(cmin.y - lpos.y, R(0)), lpos.y - cmax.y);
            R dz = std::max(std::max(cmin.z - lpos.z, R(0)), lpos.z - cmax.z);
            R padded = lrange + std::max(R(1e-4), lrange * R(1e-5));
            bool intersects = dx * dx + dy * dy + dz * dz <= padded * padded;
            bool member = ltype < R(2.5) && (ltype < R(0.5) || lrange <= R(0) || intersects);
            if (member) {
                if (count < (uint32_t)LIGHTS_PER_CELL) out[listBase + 1 + count] = (float)li;
                count++;
            }
        }
        out[listBase] = (float)(count > (uint32_t)LIGHTS_PER_CELL ? LIGHT_CELL_OVERFLOW : count);
    }
}

// Hardware bilinear on an RGBA16F texture with clamp-to-edge addressing,
// evaluated with exact weights (texel centres at i + 0.5).
inline double texel_value(uint16_t h) { return from_half(h); }
inline double texel_value(double d) { return d; }

// `atlas` holds RGBA16F texels (uint16_t) or, for the unrounded feedback of the
// adjoint checks, the same texels as doubles.
template <class R, class T> inline V3<R> bilinear_rgb(const T* atlas, uint32_t W, uint32_t H, R u, R v) {
    R x = u * R(W) - R(0.5), y = v * R(H) - R(0.5);
    R fx0 = std::floor(x), fy0 = std::floor(y);
    R fx = x - fx0, fy = y - fy0;
    long x0 = (long)fx0, y0 = (long)fy0;
    auto cl = [](long a, long n) { return a < 0 ? 0 : (a >= n ? n - 1 : a); };
    long xs[2] = {cl(x0, W), cl(x0 + 1, W)}, ys[2] = {cl(y0, H), cl(y0 + 1, H)};
    V3<R> out;
    R wxs[2] = {R(1) - fx, fx}, wys[2] = {R(1) - fy, fy};
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            const T* t = atlas + ((size_t)ys[j] * W + xs[i]) * 4;
            R w = wxs[i] * wys[j];
            out = out + V3<R>(R(texel_value(t[0])), R(texel_value(t[1])), R(texel_value(t[2]))) * w;
        }
    return out;
}

// sampleAtlas, gi_probes.js:1941-1974
template <class R, class T> V3<R> sample_atlas(const Grid& g, const T* atlas, V3<R> P, V3<R> N) {
    V3<R> cell(R(g.gridSize[0]) / std::max(R(1), R(g.res[0]) - R(1)),
               R(g.gridSize[1]) / std::max(R(1), R(g.res[1]) - R(1)),
               R(g.gridSize[2]) / std::max(R(1), R(g.res[2]) - R(1)));
    V3<R> gmin{R(g.gridMin[0]), R(g.gridMin[1]), R(g.gridMin[2])};
    V3<R> d = P - gmin;
    V3<R> gridF(d.x / std::max(cell.x, R(1e-6)), d.y / std::max(cell.y, R(1e-6)), d.z / std::max(cell.z, R(1e-6)));
    R resv[3] = {R(g.res[0]), R(g.res[1]), R(g.res[2])};
    R gf[3] = {gridF.x, gridF.y, gridF.z}, base[3], frac[3];
    for (int a = 0; a < 3; ++a) {
        base[a] = clampv(std::floor(gf[a]), R(0), std::max(resv[a] - R(2), R(0)));
        frac[a] = clampv(gf[a] - base[a], R(0), R(1));
    }
    R ou, ov;
    oct_encode(normalize(N), ou, ov);
    V3<R> acc;
    R wsum = 0;
    R W = R(g.atlasW()), H = R(g.atlasH());
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        R px = base[0] + R(dx), py = base[1] + R(dy), pz = base[2] + R(dz);
        R wx = dx ? frac[0] : R(1) - frac[0];
        R wy = dy ? frac[1] : R(1) - frac[1];
        R wz = dz ? frac[2] : R(1) - frac[2];
        R w = wx * wy * wz + R(1e-4);
        R col = px, row = pz * resv[1] + py;
        R ox = col * R(TILE) + R(BORDER) + ou * R(OCT_RES);
        R oy = row * R(TILE) + R(BORDER) + ov * R(OCT_RES);
        acc = acc + bilinear_rgb<R>(atlas, g.atlasW(), g.atlasH(), ox / W, oy / H) * w;
        wsum += w;
    }
    return acc * (R(1) / std::max(wsum, R(1e-4)));
}

// SH-9 sky on a miss, gi_probes.js:2196-2206 (THREE.SphericalHarmonics3 basis).
template <class R> V3<R> sky(const Params& P, V3<R> rd) {
    R x = rd.x, y = rd.y, z = rd.z;
    R b[9] = {R(0.282095), y * R(0.488603), z * R(0.488603), x * R(0.488603), x * y * R(1.092548),
              y * z * R(1.092548), (z * z * R(3.0) - R(1.0)) * R(0.315392), x * z * R(1.092548),
              (x * x - y * y) * R(0.546274)};
    V3<R> s;
    for (int i = 0; i < 9; ++i) s = s + V3<R>(R(P.skySH[i * 3]), R(P.skySH[i * 3 + 1]), R(P.skySH[i * 3 + 2])) * b[i];
    return V3<R>(std::max(s.x, R(0)), std::max(s.y, R(0)), std::max(s.z, R(0))) * R(P.skyIntensity);
}

template <class R> struct Tracer {
    const Scene& s;
    const Lights& L;
    const Grid& g;     // the cascade being solved
    const Grid& g0;    // cascade 0 (clustered cell lists are C0-only)
    const Params& P;
    const uint16_t* atlasPrev;  // previous upload's irradiance atlas (RGBA16F)
    Traverser<R> tr;
    // Adjoint checks: the previous atlas as unrounded doubles, and shading
    // parameters in FP64 that replace the material / light record values
    // (albedo = floats 0..2, emissive = floats 7..9, a scale of the light
    // colour 7..9). Null = use the records.
    const double* atlasPrevD = nullptr;
    const double* albedo = nullptr;
    const double* emissive = nullptr;
    const double* lightScale = nullptr;
    // Reflection lobes on (tier rough and above): hits on surfaces with no
    // diffuse energy and no emission are encoded as -(t + 2).
    bool roughEncode = false;
    // Intermediates of one hit's shading, filled when non-null (adjoint checks):
    // the unblocked lights' terms are kd (.) X[i].
    struct ShadeRecord {
        bool hit = false;
        uint32_t m = 0;
        R kdScale = 0;
        V3<R> kdr, kd, smp, bounce, hitPos, ng;
        uint32_t nLights = 0;
        uint32_t li[MAX_LIGHTS];
        V3<R> X[MAX_LIGHTS];
    };
    mutable ShadeRecord* rec = nullptr;
    Tracer(const Scene& sc, const Lights& l, const Grid& gg, const Grid& gg0, const Params& pp, const uint16_t* ap)
        : s(sc), L(l), g(gg), g0(gg0), P(pp), atlasPrev(ap), tr(sc) {}

    // shadeLight, gi_probes.js:2065-2107 (clustered) / 2130-2175 (all lights).
    void shade_light(uint32_t li, V3<R> hitPos, V3<R> ng, V3<R> kd, R traceBias, V3<R>& radiance,
                     RayOut<R>& o, const uint64_t* replayBlocked) const {
        const float* Lr = L.data + (size_t)li * LIGHT_STRIDE;
        R ltype = R(Lr[0]);
        if (!(ltype < R(2.5))) return;
        V3<R> lpos{R(Lr[1]), R(Lr[2]), R(Lr[3])}, ldir{R(Lr[4]), R(Lr[5]), R(Lr[6])};
        R eclass = R(Lr[16]);
        bool isIr = std::fabs(eclass - R(4)) < R(0.25);
        R irs = isIr ? R(P.nirGate) * R(P.nirGain) : R(1);
        V3<R> lcol = V3<R>(R(Lr[7]), R(Lr[8]), R(Lr[9])) * irs;
        if (lightScale) lcol = lcol * R(lightScale[li]);
        R lrange = R(Lr[10]), ldecay = R(Lr[11]), lcosAngle = R(Lr[12]), lcosPen = R(Lr[13]);
        bool isDir = ltype < R(0.5);
        bool isSpot = std::fabs(ltype - R(2)) < R(0.5);
        V3<R> toLight = isDir ? ldir * R(-1) : lpos - hitPos;
        R dist = isDir ? R(1e4) : std::max(length(toLight), R(1e-4));
        V3<R> wi = normalize(toLight);
        R ndl = std::max(dot(ng, wi), R(0));
        R lpeak = std::max(std::max(lcol.x, lcol.y), lcol.z);
        if (!(ndl * lpeak > R(0) && (isDir || lrange <= R(0) || dist < lrange))) return;
        bool blocked;
        if (replayBlocked) {
            blocked = (*replayBlocked >> li) & 1ull;
        } else {
            blocked = tr.any(hitPos, wi, dist - traceBias);
        }
        o.tested |= 1ull << (li & 63);
        if (blocked) { o.blocked |= 1ull << (li & 63); return; }
        R falloff = R(1) / std::max(std::pow(dist, ldecay), R(0.01));
        R rr = dist / std::max(lrange, R(1e-4));
        R rr2 = rr * rr;
        R win = clampv(R(1) - rr2 * rr2, R(0), R(1));
        R ranged = falloff * (win * win);
        R posAtten = lrange > R(0) ? ranged : falloff;
        R distAtten = isDir ? R(1) : posAtten;
        R angleCos = dot(wi, ldir) * R(-1);
        R spotAtten = clampv((angleCos - lcosAngle) / std::max(lcosPen - lcosAngle, R(1e-4)), R(0), R(1));
        R atten = distAtten * (isSpot ? spotAtten : R(1));
        V3<R> diffuse = kd * (R(1) / R(PI));
        radiance = radiance + mulv(diffuse * ndl, lcol) * atten * R(P.debugDirectScale);
        if (rec && rec->nLights < (uint32_t)MAX_LIGHTS) {
            rec->li[rec->nLights] = li;
            rec->X[rec->nLights++] = mulv(V3<R>(R(1), R(1), R(1)) * (ndl / R(PI)), lcol) * atten * R(P.debugDirectScale);
        }
    }

    // traceKernel body for one (slot, k), gi_probes.js:1977-2214.
    void trace(uint32_t slot, uint32_t k, uint32_t probeOffset, RayOut<R>& o, const Replay* rp, size_t rayIdx) const {
        uint32_t probeIndex = (probeOffset + slot) % g.probeTotal();
        V3<R> ro = probe_world_pos<R>(g, probeIndex);
        V3<R> rd = ray_dir<R>(k, g.rays, R(P.frameJitter));
        o.tested = o.blocked = 0;
        R bestT, secondT;
        int bestTri, bestInst;
        int replayFacing = -1;  // the GPU's facing decision (instance word bit 31)
        if (rp) {
            bestTri = rp->tri[rayIdx];
            uint32_t w = (uint32_t)rp->inst[rayIdx];
            bestInst = (int)(w & 0x7FFFFFFFu);
            replayFacing = (int)(w >> 31);
            secondT = R(T_MAX);
            bestT = R(T_MAX);
            if (bestTri >= 0) {
                // the FP64 parameter of the GPU's chosen triangle
                V3<R> lro = tr.inst_inv_point(bestInst, ro), lrd = tr.inst_inv_dir(bestInst, rd);
                V3<R> p0 = tr.fetch_vert(tr.tri_vert(bestTri, 0)), p1 = tr.fetch_vert(tr.tri_vert(bestTri, 1)),
                      p2 = tr.fetch_vert(tr.tri_vert(bestTri, 2));
                V3<R> e1 = p1 - p0, e2 = p2 - p0, pv = cross(lrd, e2);
                R det = dot(e1, pv);
                V3<R> tv = lro - p0, qv = cross(tv, e1);
                bestT = dot(e2, qv) * (R(1) / det);
            }
        } else {
            tr.closest(ro, rd, bestT, bestTri, bestInst, secondT);
        }
        o.tri = bestTri;
        o.inst = bestInst;
        o.secondT = secondT;
        V3<R> outRgb;
        R hitT = R(-1);
        if (bestTri >= 0) {
            hitT = bestT;
            uint32_t tri = (uint32_t)bestTri, inst = (uint32_t)bestInst;
            uint32_t m = s.triMaterial[tri];
            V3<R> p0 = tr.fetch_vert(tr.tri_vert(tri, 0)), p1 = tr.fetch_vert(tr.tri_vert(tri, 1)),
                  p2 = tr.fetch_vert(tr.tri_vert(tri, 2));
            V3<R> ngRaw = tr.inst_normal_to_world(inst, normalize(cross(p1 - p0, p2 - p0)));
            bool faceFwd = replayFacing >= 0 ? replayFacing == 1 : dot(ngRaw, rd) < R(0);
            o.facing = faceFwd ? 1 : 0;
            V3<R> ng = ngRaw * (faceFwd ? R(1) : R(-1));
            V3<R> hitPoint = ro + rd * bestT;
            R traceBias = std::max(R(g.cellMin) * R(TRACE_SURFACE_BIAS_CELL) * R(P.debugTraceBiasScale),
                                   R(RAY_EPS) * R(P.debugRayEpsScale));
            V3<R> hitPos = hitPoint + ng * traceBias;
            V3<R> baseColor(tr.mat_f(m, 0), tr.mat_f(m, 1), tr.mat_f(m, 2));
            V3<R> emis(tr.mat_f(m, 7), tr.mat_f(m, 8), tr.mat_f(m, 9));
            if (albedo) baseColor = V3<R>(R(albedo[3 * m]), R(albedo[3 * m + 1]), R(albedo[3 * m + 2]));
            if (emissive) emis = V3<R>(R(emissive[3 * m]), R(emissive[3 * m + 1]), R(emissive[3 * m + 2]));
            V3<R> radiance = emis * R(P.debugEmissiveScale);
            R metal = tr.mat_f(m, 4), transm = tr.mat_f(m, 5);
            V3<R> kdr = baseColor * R(P.debugAlbedoScale) * (R(1) - metal) * (R(1) - transm);
            V3<R> kd(clampv(kdr.x, R(0), R(0.95)), clampv(kdr.y, R(0), R(0.95)), clampv(kdr.z, R(0), R(0.95)));
            if (roughEncode) {  // gi_probes.js:2055-2062
                R diffuseEnergy = (R(1) - metal) * (R(1) - transm);
                R emissivePeak = std::max(std::max(emis.x, emis.y), emis.z);
                if (!(diffuseEnergy > R(0.02) || emissivePeak > R(1e-6))) hitT = -(bestT + R(ROUGH_UNSHADED_T_BIAS));
            }
            if (rec) {
                rec->hit = true;
                rec->m = m;
                rec->kdScale = R(P.debugAlbedoScale) * (R(1) - metal) * (R(1) - transm);
                rec->kdr = kdr;
                rec->kd = kd;
                rec->hitPos = hitPos;
                rec->ng = ng;
                rec->nLights = 0;
            }
            const uint64_t* rb = rp ? &rp->blocked[rayIdx] : nullptr;
            if (L.clustered) {
                V3<R> cellCount{R(g0.res[0]) - R(1), R(g0.res[1]) - R(1), R(g0.res[2]) - R(1)};
                V3<R> cellSize(R(g0.gridSize[0]) / cellCount.x, R(g0.gridSize[1]) / cellCount.y,
                               R(g0.gridSize[2]) / cellCount.z);
                V3<R> rel = hitPos - V3<R>(R(g0.gridMin[0]), R(g0.gridMin[1]), R(g0.gridMin[2]));
                V3<R> cf(std::floor(rel.x / cellSize.x), std::floor(rel.y / cellSize.y), std::floor(rel.z / cellSize.z));
                bool outside = cf.x < R(0) || cf.y < R(0) || cf.z < R(0) || cf.x >= cellCount.x ||
                               cf.y >= cellCount.y || cf.z >= cellCount.z;
                uint32_t cx = (uint32_t)clampv(cf.x, R(0), cellCount.x - R(1));
                uint32_t cy = (uint32_t)clampv(cf.y, R(0), cellCount.y - R(1));
                uint32_t cz = (uint32_t)clampv(cf.z, R(0), cellCount.z - R(1));
                uint32_t cellsX = g0.res[0] - 1, cellsY = g0.res[1] - 1;
                uint32_t cellIndex = cz * (cellsX * cellsY) + cy * cellsX + cx;
                size_t listBase = (size_t)MAX_LIGHTS * LIGHT_STRIDE + (size_t)cellIndex * LIGHT_CELL_STRIDE;
                uint32_t listCount = (uint32_t)L.data[listBase];
                if (outside || listCount > (uint32_t)LIGHTS_PER_CELL) {
                    for (uint32_t li = 0; li < L.lightCount; ++li)
                        shade_light(li, hitPos, ng, kd, traceBias, radiance, o, rb);
                } else {
                    for (uint32_t i = 0; i < listCount; ++i)
                        shade_light((uint32_t)L.data[listBase + 1 + i], hitPos, ng, kd, traceBias, radiance, o, rb);
                }
            } else {
                for (uint32_t li = 0; li < L.lightCount; ++li)
                    shade_light(li, hitPos, ng, kd, traceBias, radiance, o, rb);
            }
            V3<R> smp = atlasPrevD ? sample_atlas<R>(g, atlasPrevD, hitPos, ng) : sample_atlas<R>(g, atlasPrev, hitPos, ng);
            V3<R> bounce = mulv(smp, kd) * (R(1) / R(PI));
            if (rec) {
                rec->smp = smp;
                rec->bounce = bounce;
            }
            R bl = luma(bounce);
            R roll = R(P.radianceClamp) / std::max(std::max(R(P.radianceClamp), bl), R(1e-6));
            radiance = radiance + bounce * roll * R(P.debugBounceScale);
            outRgb = radiance;
        } else {
            if (rec) rec->hit = false;
            outRgb = sky<R>(P, rd);
        }
        o.rgb[0] = outRgb.x;
        o.rgb[1] = outRgb.y;
        o.rgb[2] = outRgb.z;
        o.hitT = hitT;
    }
};

// Texel <- source lane of the canonical mirrored gutter, gi_probes.js:2816-2839.
inline int gutter_source_lane(int lane) {
    const int edge = TILE - 1, lo = BORDER, hi = BORDER + OCT_RES - 1;
    int lx = lane % TILE, ly = lane / TILE;
    bool onLeft = lx == 0, onRight = lx == edge, onTop = ly == 0, onBottom = ly == edge;
    bool colB = onLeft || onRight, rowB = onTop || onBottom, corner = colB && rowB;
    int sx = corner ? (onLeft ? hi : lo) : (rowB ? edge - lx : (colB ? (onLeft ? lo : hi) : lx));
    int sy = corner ? (onTop ? hi : lo) : (rowB ? (onTop ? lo : hi) : (colB ? edge - ly : ly));
    return (sy - BORDER) * OCT_RES + (sx - BORDER);
}

// blendKernel (gi_probes.js:2317-2532) for one probe slot: reads the slot's rays
// (rgb + hitT, 4 per ray), updates the irradiance (4/texel) and depth (2/texel)
// histories of its 36 interior texels.
// emitterVisKernel's sample for (probe, emitter) (gi_probes.js:2216-2260): a
// shadow ray from the probe to a point of the emitter's disk (a sin hash of
// the probe, the emitter and the epoch seed, evaluated in float32 as the GPU
// does), 1 when unblocked. With sourceRadius 0 the point is the centre.
template <class R> R emitter_sample(const Scene& s, const Lights& L, const Grid& g, const Params& P, uint32_t probeIndex,
                                    uint32_t e) {
    const float* rec = L.data + (size_t)(L.emitterBase + e) * LIGHT_STRIDE;
    const V3<R> ro = probe_world_pos<R>(g, probeIndex);
    const V3<R> center = V3<R>(R(rec[1]), R(rec[2]), R(rec[3]));
    R sourceRadius = std::max(R(rec[14]), R(0));
    V3<R> axis = center - ro;
    R dist = length(axis);
    if (!(dist > std::max(sourceRadius, R(1e-3)))) return R(0);
    V3<R> d = axis * (R(1) / dist);
    V3<R> up = std::fabs(d.y) < R(0.999) ? V3<R>(R(0), R(1), R(0)) : V3<R>(R(1), R(0), R(0));
    V3<R> tangent = normalize(cross(up, d));
    V3<R> bitangent = cross(d, tangent);
    const float seed = (float(probeIndex) * 12.9898f + float(e) * 78.233f) + float(P.emitterVisSeed) * 37.719f;
    const float h0 = std::sin(seed) * 43758.5453f;
    const float h1 = std::sin(seed + 19.19f) * 24634.6345f;
    const float u = h0 - std::floor(h0), v = h1 - std::floor(h1);
    R diskRadius = std::sqrt(R(u)) * sourceRadius;
    R diskAngle = R(v) * R(2.0 * PI);
    V3<R> target = center + (tangent * (std::cos(diskAngle) * diskRadius) + bitangent * (std::sin(diskAngle) * diskRadius));
    V3<R> sdir = normalize(target - ro);
    R traceBias = std::max(R(g.cellMin) * R(TRACE_SURFACE_BIAS_CELL) * R(P.debugTraceBiasScale),
                           R(RAY_EPS) * R(P.debugRayEpsScale));
    Traverser<R> tr(s);
    bool blocked = tr.any(ro, sdir, std::max(dist - sourceRadius - traceBias, R(1e-4)));
    return blocked ? R(0) : R(1);
}

// The emitters a blend injects as virtual rays (injectEmitterVirtualRays,
// gi_probes.js:2262-2310): the records and this probe's visibility per emitter.
template <class R> struct EmitterInject {
    const Lights* L = nullptr;
    const R* vis = nullptr;  // probeTotal x GI_EMITTER_INJECT_CAP
};

// Reflection lobe state of one cascade (REFLECTION_QUALITY_TIERS,
// gi_probes.js:60-75; buffers 1796-1840): tier 1 rough, 2 high, 3 ultra.
template <class R> struct Reflect {
    uint32_t tier = 0;
    R* roughSpec = nullptr;         // probeTotal x 64 texels x 4 (rgb, coverage)
    uint16_t* roughAtlas = nullptr; // RGBA16F, the irradiance atlas layout
    R* glossyNum = nullptr;         // probeTotal x glossyTile^2 x 4
    R* glossyDen = nullptr;         // probeTotal x glossyTile^2
    uint16_t* glossyAtlas = nullptr;
    uint32_t glossyPhase = 0;
    uint32_t oct() const { return tier == 2 ? 8u : tier == 3 ? 16u : 1u; }
    uint32_t tile() const { return tier >= 2 ? oct() + 2u * BORDER : 1u; }
    uint32_t interval() const { return tier == 2 ? 2u : tier == 3 ? 1u : 0u; }
    // glossy tiles packed near-square (gi_probes.js:3107-3110)
    static uint32_t tiles_x(uint32_t probeTotal) {
        return std::max(1u, (uint32_t)std::ceil(std::sqrt((double)probeTotal)));
    }
};

template <class R> void blend_probe(const Grid& g, const Params& P, const R* rays, uint32_t probeIndex, R* irr, R* depth,
                                    const EmitterInject<R>* em = nullptr, Reflect<R>* rf = nullptr) {
    const bool rough = rf && rf->tier >= 1;
    // a true miss feeds the lobe only with the explicit sky fallback (gi_probes.js:2361-2367)
    const R skyValid = R(P.reflectionSkyFallback) * R(P.skyConfigured) * (P.skyIntensity > 0 ? R(1) : R(0));
    const uint32_t N = g.rays;
    std::vector<V3<R>> dirs(N);
    for (uint32_t k = 0; k < N; ++k) dirs[k] = ray_dir<R>(k, N, R(P.frameJitter));
    for (int lane = 0; lane < OCT_RES * OCT_RES; ++lane) {
        int lx = lane % OCT_RES + BORDER, ly = lane / OCT_RES + BORDER;
        int local = ly * TILE + lx;
        R u = (R(lx) - R(BORDER) + R(0.5)) / R(OCT_RES);
        R v = (R(ly) - R(BORDER) + R(0.5)) / R(OCT_RES);
        V3<R> dir = oct_decode(u, v);
        V3<R> acc, sAcc;
        R wsum = 0, dAcc = 0, dAcc2 = 0, dwsum = 0, lAcc = 0, lAcc2 = 0, sHit = 0, sWsum = 0;
        for (uint32_t k = 0; k < N; ++k) {
            const R* rr = rays + (size_t)k * 4;
            V3<R> rrgb(rr[0], rr[1], rr[2]);
            R hitT = rr[3];
            R cd = std::max(dot(dir, dirs[k]), R(0));
            R cw = std::pow(cd, std::max(R(P.debugCosinePower), R(1e-4)));
            acc = acc + rrgb * cw;
            wsum += cw;
            R rl = luma(rrgb);
            lAcc += rl * cw;
            lAcc2 += rl * rl * cw;
            bool roughUnshaded = hitT < R(-1.5);
            R decoded = roughUnshaded ? -hitT - R(2) : hitT;
            R rdist = hitT == R(-1) ? R(g.maxDist) : decoded;
            R dw = std::pow(cw, R(P.depthSharpness));
            dAcc += rdist * dw;
            dAcc2 += rdist * rdist * dw;
            dwsum += dw;
            if (rough) {  // power-8 lobe (gi_probes.js:2388-2404)
                R cd2 = cd * cd, cd4 = cd2 * cd2, sw = cd4 * cd4;
                R valid = hitT >= R(0) ? R(1) : (hitT == R(-1) ? skyValid : R(0));
                sAcc = sAcc + rrgb * sw * valid;
                sHit += sw * valid;
                sWsum += sw;
            }
        }
        if (em && em->L && em->L->emitterCount) {
            // each emitter as kVirtual rays toward its centre, radiance x visibility
            const V3<R> ro = probe_world_pos<R>(g, probeIndex);
            for (uint32_t e = 0; e < em->L->emitterCount; ++e) {
                const float* rec = em->L->data + (size_t)(em->L->emitterBase + e) * LIGHT_STRIDE;
                const V3<R> center = V3<R>(R(rec[1]), R(rec[2]), R(rec[3]));
                R sourceRadius = std::max(R(rec[14]), R(0));
                V3<R> axis = center - ro;
                R dist = length(axis);
                if (!(dist > std::max(sourceRadius, R(1e-3)))) continue;
                V3<R> d = axis * (R(1) / dist);
                R projArea = std::max(R(rec[15]), R(0));
                R Omega = std::min(R(2.0 * PI), projArea / (dist * dist));
                R kVirtual = std::min(R(N), R(N) * Omega / R(4.0 * PI));
                R vis = em->vis[(size_t)probeIndex * GI_EMITTER_INJECT_CAP + e];
                V3<R> Lc = V3<R>(R(rec[7]), R(rec[8]), R(rec[9])) * vis;
                R cd = std::max(dot(dir, d), R(0));
                R w = std::pow(cd, std::max(R(P.debugCosinePower), R(1e-4)));
                R wk = w * kVirtual;
                acc = acc + Lc * wk;
                wsum += wk;
                R lum = luma(Lc);
                lAcc += lum * wk;
                lAcc2 += lum * lum * wk;
                if (rough) {
                    R cd2 = cd * cd, cd4 = cd2 * cd2;
                    R swk = cd4 * cd4 * kVirtual;
                    sAcc = sAcc + Lc * swk;
                    sHit += swk;
                    sWsum += swk;
                }
            }
        }
        R wden = std::max(wsum, R(1e-4));
        V3<R> meanRad(acc.x / wden, acc.y / wden, acc.z / wden);
        R curL = lAcc / wden, curM2 = lAcc2 / wden;
        R dden = std::max(dwsum, R(1e-4));
        R meanR = dAcc / dden, meanR2 = dAcc2 / dden;

        size_t ib = ((size_t)probeIndex * TILE * TILE + local) * 4;
        V3<R> prev(irr[ib], irr[ib + 1], irr[ib + 2]);
        bool wasBlack = (prev.x + prev.y + prev.z) < R(1e-6);
        R prevL = luma(prev);
        R prevM2 = irr[ib + 3];
        R prevVar = std::max(prevM2 - prevL * prevL, R(0));
        R curVar = std::max(curM2 - curL * curL, R(0));
        R lumRef = std::max(std::max(curL, prevL), R(0));
        R varFloor = R(P.debugTempVarEps) + lumRef * lumRef * R(P.debugTempVarRel);
        R sigma = std::sqrt(prevVar + curVar + varFloor);
        R deltaL = curL - prevL;
        R absDelta = std::fabs(deltaL);
        R s0 = sigma * R(P.debugTempChangeSigma0);
        R s1 = sigma * std::max(R(P.tempChangeSigma1), R(P.debugTempChangeSigma0) + R(0.01));
        R changeW = clampv((absDelta - s0) / std::max(s1 - s0, R(1e-6)), R(0), R(1));
        R H = R(P.hysteresis);
        R rawNoiseH = H + (R(1) - H) * R(P.debugTempNoiseHBoost);
        R rawChangeH = std::max(H - R(P.tempChangeHDrop), R(P.debugTempMinChangeH));
        R rawHEff = mixv(rawNoiseH, rawChangeH, changeW);
        R hEff = std::pow(clampv(rawHEff, R(1e-6), R(1)), R(P.hysteresisExponent));
        R h = wasBlack ? R(0) : hEff;
        R band = std::sqrt(prevVar + varFloor) * R(P.tempClampSigma);
        R clampScale = std::min(R(1), band / std::max(absDelta, R(1e-6)));
        V3<R> clipped = prev + (meanRad - prev) * clampScale;
        V3<R> candidate = wasBlack ? meanRad : clipped;
        V3<R> blended = mix3(candidate, prev, h);
        irr[ib] = blended.x;
        irr[ib + 1] = blended.y;
        irr[ib + 2] = blended.z;
        irr[ib + 3] = mixv(curM2, prevM2, h);

        size_t db = ((size_t)probeIndex * TILE * TILE + local) * 2;
        R dpx = depth[db], dpy = depth[db + 1];
        bool dWasZero = dpx < R(1e-6);
        if (rough) {  // rough history: steady / noisy reference retention (gi_probes.js:2478-2484, 2505-2522)
            R steadyH = std::pow(clampv(rawNoiseH, R(1e-6), R(1)), R(P.hysteresisExponent));
            R sh = dWasZero ? R(0) : steadyH;
            R sDen = std::max(sWsum, R(1e-4));
            R sCur[4] = {sAcc.x / sDen, sAcc.y / sDen, sAcc.z / sDen, clampv(sHit / sDen, R(0), R(1))};
            R* sp = rf->roughSpec + ib;
            for (int c = 0; c < 4; ++c) sp[c] = mixv(sCur[c], sp[c], sh);
        }
        R rawDepthH = clampv(H * R(P.debugDepthHistoryScale), R(0), R(0.999));
        R depthH = std::pow(std::max(rawDepthH, R(1e-6)), R(P.hysteresisExponent));
        R dh = dWasZero ? R(0) : depthH;
        depth[db] = mixv(meanR, dpx, dh);
        depth[db + 1] = mixv(meanR2, dpy, dh);
    }
}

// uploadKernel (gi_probes.js:2737-2846) for one probe: 3x3 bilateral filter of
// the irradiance history and the mirrored-gutter RGBA16F tile writes. When
// preRound != nullptr, the unrounded RGB of the 36 interior texels (the value
// that the fp16 store rounds) is also returned, probe-major, 3 per texel.
template <class R> void upload_probe(const Grid& g, const Params& P, uint32_t probeIndex, const R* irr, const R* depth,
                                     uint16_t* atlas, uint16_t* depthAtlas, R* preRound, const Reflect<R>* rf = nullptr) {
    R cacheI[36][3], cacheD[36][2];
    size_t probeBase = (size_t)probeIndex * TILE * TILE;
    for (int lane = 0; lane < OCT_RES * OCT_RES; ++lane) {
        int sx = lane % OCT_RES + BORDER, sy = lane / OCT_RES + BORDER;
        size_t pt = probeBase + sy * TILE + sx;
        V3<R> eC(irr[pt * 4], irr[pt * 4 + 1], irr[pt * 4 + 2]);
        R lumaC = luma(eC);
        R varC = std::max(irr[pt * 4 + 3] - lumaC * lumaC, R(0));
        V3<R> facc;
        R fwsum = 0;
        R smW = R(1) + R(P.filterSmooth) * R(6);
        R kEff = R(GI_FILTER_K) * smW * R(P.debugFilterKScale);
        R relEff = R(GI_FILTER_REL) * smW * R(P.debugFilterRelScale);
        for (int jy = -1; jy <= 1; ++jy)
            for (int jx = -1; jx <= 1; ++jx) {
                R gw = R(std::exp(-(double)(jx * jx + jy * jy) * 0.5));
                int nx = std::min(std::max(sx + jx, BORDER), BORDER + OCT_RES - 1);
                int ny = std::min(std::max(sy + jy, BORDER), BORDER + OCT_RES - 1);
                size_t nIb = (probeBase + ny * TILE + nx) * 4;
                V3<R> en(irr[nIb], irr[nIb + 1], irr[nIb + 2]);
                R dLum = luma(en) - lumaC;
                R den = std::max(varC * kEff + std::max(R(GI_FILTER_EPS) * R(P.debugFilterEpsScale), lumaC * lumaC * relEff), R(1e-8));
                R es = std::exp(dLum * dLum / den * R(-1));
                R w = gw * es;
                facc = facc + en * w;
                fwsum += w;
            }
        R fden = std::max(fwsum, R(1e-4));
        V3<R> filtered(facc.x / fden, facc.y / fden, facc.z / fden);
        V3<R> outc = mix3(eC, filtered, R(P.filterStrength));
        cacheI[lane][0] = outc.x; cacheI[lane][1] = outc.y; cacheI[lane][2] = outc.z;
        cacheD[lane][0] = depth[pt * 2];
        cacheD[lane][1] = depth[pt * 2 + 1];
        if (preRound) {
            R* pr = preRound + ((size_t)probeIndex * 36 + lane) * 3;
            pr[0] = outc.x; pr[1] = outc.y; pr[2] = outc.z;
        }
    }
    uint32_t rx = g.res[0], ry = g.res[1];
    uint32_t col = probeIndex % rx;
    uint32_t row = (probeIndex / (rx * ry)) * ry + (probeIndex / rx) % ry;
    uint32_t W = g.atlasW();
    for (int lane = 0; lane < TILE * TILE; ++lane) {
        int lx = lane % TILE, ly = lane / TILE;
        int src = gutter_source_lane(lane);
        size_t t = ((size_t)(row * TILE + ly) * W + col * TILE + lx) * 4;
        atlas[t] = to_half(cacheI[src][0]);
        atlas[t + 1] = to_half(cacheI[src][1]);
        atlas[t + 2] = to_half(cacheI[src][2]);
        atlas[t + 3] = to_half(1.0);
        depthAtlas[t] = to_half(cacheD[src][0]);
        depthAtlas[t + 1] = to_half(cacheD[src][1]);
        depthAtlas[t + 2] = to_half(0.0);
        depthAtlas[t + 3] = to_half(1.0);
        if (rf && rf->tier >= 1) {  // the rough history, unfiltered (gi_probes.js:2789-2795, 2841-2843)
            int ssx = src % OCT_RES + BORDER, ssy = src / OCT_RES + BORDER;
            const R* sp = rf->roughSpec + (probeBase + ssy * TILE + ssx) * 4;
            for (int c = 0; c < 4; ++c) rf->roughAtlas[t + c] = to_half(sp[c]);
        }
    }
}

// glossyKernel (gi_probes.js:2538-2686) for one probe: the power-64 lobe on the
// glossy tile (glossyOct^2 texels and a mirrored one-texel gutter, each gutter
// texel evaluated at its source texel's direction), the per-ray-mean numerator
// and support histories and the resolved RGBA16F glossy atlas. Tier high
// resolves the texels with local % 2 == glossyPhase.
template <class R> void glossy_probe(const Grid& g, const Params& P, const R* rays, uint32_t probeIndex,
                                     Reflect<R>& rf, const EmitterInject<R>* em = nullptr) {
    const uint32_t N = g.rays, tile = rf.tile(), oct = rf.oct(), interval = rf.interval();
    std::vector<V3<R>> dirs(N);
    for (uint32_t k = 0; k < N; ++k) dirs[k] = ray_dir<R>(k, N, R(P.frameJitter));
    const R skyValid = R(P.reflectionSkyFallback) * R(P.skyConfigured) * (P.skyIntensity > 0 ? R(1) : R(0));
    const uint32_t tilesX = Reflect<R>::tiles_x(g.probeTotal());
    const uint32_t atlasW = tilesX * tile;
    auto pow64 = [](R c) { R c2 = c * c, c4 = c2 * c2, c8 = c4 * c4, c16 = c8 * c8, c32 = c16 * c16; return c32 * c32; };
    for (uint32_t local = 0; local < tile * tile; ++local) {
        if (interval > 1 && local % interval != rf.glossyPhase) continue;
        const int lx = (int)(local % tile), ly = (int)(local / tile);
        const int edge = (int)tile - 1, lo = BORDER, hi = BORDER + (int)oct - 1;
        bool onLeft = lx == 0, onRight = lx == edge, onTop = ly == 0, onBottom = ly == edge;
        bool colB = onLeft || onRight, rowB = onTop || onBottom, corner = colB && rowB;
        int sx = corner ? (onLeft ? hi : lo) : (rowB ? edge - lx : (colB ? (onLeft ? lo : hi) : lx));
        int sy = corner ? (onTop ? hi : lo) : (rowB ? (onTop ? lo : hi) : (colB ? edge - ly : ly));
        R u = (R(sx) - R(BORDER) + R(0.5)) / R(oct);
        R v = (R(sy) - R(BORDER) + R(0.5)) / R(oct);
        V3<R> dir = oct_decode(u, v);
        V3<R> gAcc;
        R gHit = 0, gWsum = 0;
        for (uint32_t k = 0; k < N; ++k) {
            const R* rr = rays + (size_t)k * 4;
            R hitT = rr[3];
            R gw = pow64(std::max(dot(dir, dirs[k]), R(0)));
            R valid = hitT >= R(0) ? R(1) : (hitT == R(-1) ? skyValid : R(0));
            gAcc = gAcc + V3<R>(rr[0], rr[1], rr[2]) * gw * valid;
            gHit += gw * valid;
            gWsum += gw;
        }
        if (em && em->L && em->L->emitterCount) {
            const V3<R> ro = probe_world_pos<R>(g, probeIndex);
            for (uint32_t e = 0; e < em->L->emitterCount; ++e) {
                const float* rec = em->L->data + (size_t)(em->L->emitterBase + e) * LIGHT_STRIDE;
                const V3<R> center = V3<R>(R(rec[1]), R(rec[2]), R(rec[3]));
                R sourceRadius = std::max(R(rec[14]), R(0));
                V3<R> axis = center - ro;
                R dist = length(axis);
                if (!(dist > std::max(sourceRadius, R(1e-3)))) continue;
                V3<R> d = axis * (R(1) / dist);
                R Omega = std::min(R(2.0 * PI), std::max(R(rec[15]), R(0)) / (dist * dist));
                R kVirtual = std::min(R(N), R(N) * Omega / R(4.0 * PI));
                R vis = em->vis[(size_t)probeIndex * GI_EMITTER_INJECT_CAP + e];
                V3<R> Lc = V3<R>(R(rec[7]), R(rec[8]), R(rec[9])) * vis;
                R wk = pow64(std::max(dot(dir, d), R(0))) * kVirtual;
                gAcc = gAcc + Lc * wk;
                gWsum += wk;
                gHit += wk;
            }
        }
        const size_t gt = (size_t)probeIndex * tile * tile + local;
        R* num = rf.glossyNum + gt * 4;
        R& den = rf.glossyDen[gt];
        // the reference forms 1 / raysPerProbe in double and stores it as a float uniform
        R invRays = R(float(1.0 / double(N)));
        R curNum[4] = {gAcc.x * invRays, gAcc.y * invRays, gAcc.z * invRays, gHit * invRays};
        R curDen = gWsum * invRays;
        bool empty = den < R(1e-6);
        R H = R(P.hysteresis);
        R refH = H + (R(1) - H) * R(P.debugTempNoiseHBoost);
        R glossyH = std::pow(clampv(refH, R(1e-6), R(1)), R(P.hysteresisExponent) * R(interval));
        R gh = empty ? R(0) : glossyH;
        for (int c = 0; c < 4; ++c) num[c] = mixv(curNum[c], num[c], gh);
        den = std::max(mixv(curDen, den, gh), R(1e-6));
        uint32_t col = probeIndex % tilesX, row = probeIndex / tilesX;
        size_t t = ((size_t)(row * tile + ly) * atlasW + col * tile + lx) * 4;
        rf.glossyAtlas[t] = to_half(num[0] / den);
        rf.glossyAtlas[t + 1] = to_half(num[1] / den);
        rf.glossyAtlas[t + 2] = to_half(num[2] / den);
        rf.glossyAtlas[t + 3] = to_half(clampv(num[3] / den, R(0), R(1)));
    }
}

}  // namespace orc
