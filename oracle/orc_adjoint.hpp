// orc_adjoint.hpp — FP64 restatement of the differentiable solve sequence and
// its reverse pass: `solves` feedback solves of one cascade (trace replayed
// from fixed hit records and shadow bits, shade, blend, upload) from a cleared
// history, the loss sum (E - target)^2 over the interior irradiance texels of
// the last solve, and the gradient of that loss with respect to per-material
// albedo and emissive and a per-light colour scale. The forward is the
// oracle's own restatement (Tracer::trace, blend_probe, upload_probe,
// gi_probes.js:1977-2214, 2317-2532, 2737-2846) with the parameters given in
// FP64; the reverse pass differentiates it by hand, holding every select at
// the side the forward value chose. With roundAtlas the atlas a later solve
// reads is rounded to binary16 as the library stores it, and the gradient
// passes straight through that rounding; without, the feedback is exact and
// central differences of the forward agree with the reverse pass to O(h^2).
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
#pragma once
#include "orc_probes.hpp"

#include <atomic>
#include <thread>

namespace orc {

struct AdjProblem {
    const Scene* sc = nullptr;
    const Lights* L = nullptr;
    Grid g;
    Params P;
    const int32_t* tri = nullptr;       // per ray, -1 = miss (the same records every solve)
    const int32_t* inst = nullptr;      // instance slot | facing << 31
    const uint64_t* blocked = nullptr;  // per ray: lights whose shadow ray was blocked
    uint32_t solves = 2;
    bool roundAtlas = true;
    uint32_t materialCount = 0, lightCount = 0;
    const double* albedo = nullptr;     // materialCount x 3
    const double* emissive = nullptr;   // materialCount x 3
    const double* lightScale = nullptr; // lightCount
    int threads = 1;
};

struct AdjTape {
    std::vector<std::vector<double>> hist;   // solves + 1 histories (probes x 64 x RGBM)
    std::vector<std::vector<double>> atlas;  // the atlas each solve's bounce reads (W x H x RGBA)
    std::vector<double> E;                   // last solve's upload output, probes x 36 x 3
};

template <class F> inline void adj_parallel(size_t n, int threads, F&& f) {
    if (threads <= 1 || n < 64) {
        for (size_t i = 0; i < n; ++i) f(i, 0);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t)
        ts.emplace_back([&, t] {
            for (;;) {
                size_t b = next.fetch_add(32);
                if (b >= n) break;
                for (size_t i = b, e = std::min(n, b + 32); i < e; ++i) f(i, t);
            }
        });
    for (auto& th : ts) th.join();
}

inline Tracer<double> adj_tracer(const AdjProblem& A, const double* atlasPrev) {
    Tracer<double> tc(*A.sc, *A.L, A.g, A.g, A.P, nullptr);
    tc.atlasPrevD = atlasPrev;
    tc.albedo = A.albedo;
    tc.emissive = A.emissive;
    tc.lightScale = A.lightScale;
    return tc;
}

inline void adj_rays(const AdjProblem& A, const double* atlasPrev, std::vector<double>& rays) {
    const uint32_t N = A.g.rays;
    const size_t nr = (size_t)A.g.probeTotal() * N;
    rays.assign(nr * 4, 0.0);
    Replay rp{A.tri, A.inst, A.blocked};
    adj_parallel(nr, A.threads, [&](size_t i, int) {
        Tracer<double> tc = adj_tracer(A, atlasPrev);
        RayOut<double> o;
        tc.trace((uint32_t)(i / N), (uint32_t)(i % N), 0, o, &rp, i);
        for (int c = 0; c < 3; ++c) rays[i * 4 + c] = o.rgb[c];
        rays[i * 4 + 3] = o.hitT;
    });
}

// Forward: fills the tape; returns the loss when target != nullptr.
inline double adj_forward(const AdjProblem& A, AdjTape& T, const double* target) {
    const Grid& g = A.g;
    const uint32_t probes = g.probeTotal(), N = g.rays, W = g.atlasW(), H = g.atlasH();
    std::vector<double> irr((size_t)probes * 64 * 4, 0.0), depth((size_t)probes * 64 * 2, 0.0);
    std::vector<double> atlas((size_t)W * H * 4, 0.0);
    for (size_t t = 0; t < (size_t)W * H; ++t) atlas[t * 4 + 3] = 1.0;  // clearAtlasKernel: (0, 0, 0, 1)
    std::vector<uint16_t> a16((size_t)W * H * 4), d16((size_t)W * H * 4);
    std::vector<double> pre((size_t)probes * 36 * 3), rays;
    T.hist.clear();
    T.atlas.clear();
    for (uint32_t s = 0; s < A.solves; ++s) {
        T.hist.push_back(irr);
        T.atlas.push_back(atlas);
        adj_rays(A, atlas.data(), rays);
        adj_parallel(probes, A.threads, [&](size_t p, int) {
            blend_probe<double>(g, A.P, rays.data() + p * N * 4, (uint32_t)p, irr.data(), depth.data());
        });
        adj_parallel(probes, A.threads, [&](size_t p, int) {
            upload_probe<double>(g, A.P, (uint32_t)p, irr.data(), depth.data(), a16.data(), d16.data(), pre.data());
        });
        for (uint32_t p = 0; p < probes; ++p) {
            uint32_t col = p % g.res[0];
            uint32_t row = (p / (g.res[0] * g.res[1])) * g.res[1] + (p / g.res[0]) % g.res[1];
            for (int lane = 0; lane < TILE * TILE; ++lane) {
                int src = gutter_source_lane(lane);
                size_t t = ((size_t)(row * TILE + lane / TILE) * W + col * TILE + lane % TILE) * 4;
                for (int c = 0; c < 3; ++c) {
                    double v = pre[((size_t)p * 36 + src) * 3 + c];
                    atlas[t + c] = A.roundAtlas ? from_half(to_half(v)) : v;
                }
                atlas[t + 3] = 1.0;
            }
        }
    }
    T.hist.push_back(irr);
    T.E = pre;
    double loss = 0.0;
    if (target)
        for (size_t i = 0; i < pre.size(); ++i) loss += (pre[i] - target[i]) * (pre[i] - target[i]);
    return loss;
}

// sampleAtlas as 32 weighted texel taps: sample = sum_i wt[i] * atlas[idx[i]]
// (gi_probes.js:1941-1974 with the clamp-to-edge bilinear of bilinear_rgb).
inline void adj_atlas_taps(const Grid& g, V3<double> P, V3<double> N, size_t* idx, double* wt) {
    V3<double> cell(g.gridSize[0] / std::max(1.0, double(g.res[0]) - 1.0),
                    g.gridSize[1] / std::max(1.0, double(g.res[1]) - 1.0),
                    g.gridSize[2] / std::max(1.0, double(g.res[2]) - 1.0));
    double gf[3] = {(P.x - g.gridMin[0]) / std::max(cell.x, 1e-6), (P.y - g.gridMin[1]) / std::max(cell.y, 1e-6),
                    (P.z - g.gridMin[2]) / std::max(cell.z, 1e-6)};
    double base[3], frac[3];
    for (int a = 0; a < 3; ++a) {
        base[a] = clampv(std::floor(gf[a]), 0.0, std::max(double(g.res[a]) - 2.0, 0.0));
        frac[a] = clampv(gf[a] - base[a], 0.0, 1.0);
    }
    double ou, ov;
    oct_encode(normalize(N), ou, ov);
    const uint32_t Wt = g.atlasW(), Ht = g.atlasH();
    const double W = Wt, H = Ht;
    double wsum = 0.0;
    auto cl = [](long a, long n) { return a < 0 ? 0 : (a >= n ? n - 1 : a); };
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        double px = base[0] + dx, py = base[1] + dy, pz = base[2] + dz;
        double w = (dx ? frac[0] : 1.0 - frac[0]) * (dy ? frac[1] : 1.0 - frac[1]) * (dz ? frac[2] : 1.0 - frac[2]) + 1e-4;
        double row = pz * double(g.res[1]) + py;
        double ox = px * TILE + BORDER + ou * OCT_RES, oy = row * TILE + BORDER + ov * OCT_RES;
        double x = (ox / W) * W - 0.5, y = (oy / H) * H - 0.5;
        double fx0 = std::floor(x), fy0 = std::floor(y), fx = x - fx0, fy = y - fy0;
        long x0 = (long)fx0, y0 = (long)fy0;
        long xs[2] = {cl(x0, Wt), cl(x0 + 1, Wt)}, ys[2] = {cl(y0, Ht), cl(y0 + 1, Ht)};
        double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy};
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) {
                idx[4 * i + 2 * j + k] = (size_t)ys[j] * Wt + xs[k];
                wt[4 * i + 2 * j + k] = w * wx[k] * wy[j];
            }
        wsum += w;
    }
    const double inv = 1.0 / std::max(wsum, 1e-4);
    for (int i = 0; i < 32; ++i) wt[i] *= inv;
}

// Reverse of upload_probe for one probe: gE (36 x 3) -> gH (64 x RGBM, added).
inline void adj_upload_bwd(const Params& P, const double* H, const double* gE, double* gH) {
    const double smW = 1.0 + P.filterSmooth * 6.0;
    const double kEff = GI_FILTER_K * smW * P.debugFilterKScale, relEff = GI_FILTER_REL * smW * P.debugFilterRelScale;
    const double epsF = GI_FILTER_EPS * P.debugFilterEpsScale, s = P.filterStrength;
    auto at = [](int sx, int sy) { return (size_t)((sy + BORDER) * TILE + sx + BORDER); };
    for (int lane = 0; lane < 36; ++lane) {
        const int sx = lane % OCT_RES, sy = lane / OCT_RES;
        const double* c4 = H + at(sx, sy) * 4;
        V3<double> eC(c4[0], c4[1], c4[2]);
        double lumaC = luma(eC), varRaw = c4[3] - lumaC * lumaC, varC = std::max(varRaw, 0.0);
        double inner = std::max(epsF, lumaC * lumaC * relEff), denRaw = varC * kEff + inner;
        double den = std::max(denRaw, 1e-8);
        V3<double> facc;
        double fw = 0.0, w[9], dl[9];
        size_t nb[9];
        for (int q = 0; q < 9; ++q) {
            int jx = q % 3 - 1, jy = q / 3 - 1;
            double gw = std::exp(-(double)(jx * jx + jy * jy) * 0.5);
            int nx = std::min(std::max(sx + jx, 0), OCT_RES - 1), ny = std::min(std::max(sy + jy, 0), OCT_RES - 1);
            nb[q] = at(nx, ny);
            V3<double> en(H[nb[q] * 4], H[nb[q] * 4 + 1], H[nb[q] * 4 + 2]);
            dl[q] = luma(en) - lumaC;
            w[q] = gw * std::exp(-dl[q] * dl[q] / den);
            facc = facc + en * w[q];
            fw += w[q];
        }
        double fden = std::max(fw, 1e-4);
        V3<double> g(gE[lane * 3], gE[lane * 3 + 1], gE[lane * 3 + 2]);
        V3<double> gEC = g * (1.0 - s), gFilt = g * s, gFacc = gFilt * (1.0 / fden);
        double gFw = fw > 1e-4 ? -dot(gFilt, facc) / (fden * fden) : 0.0;
        double gDen = 0.0, gLumaC = 0.0;
        for (int q = 0; q < 9; ++q) {
            V3<double> en(H[nb[q] * 4], H[nb[q] * 4 + 1], H[nb[q] * 4 + 2]);
            double gW = dot(gFacc, en) + gFw;
            double gq = -gW * w[q];
            double gDl = gq * 2.0 * dl[q] / den;
            gDen -= gq * dl[q] * dl[q] / (den * den);
            V3<double> add = gFacc * w[q] + V3<double>(0.2126, 0.7152, 0.0722) * gDl;
            gH[nb[q] * 4] += add.x;
            gH[nb[q] * 4 + 1] += add.y;
            gH[nb[q] * 4 + 2] += add.z;
            gLumaC -= gDl;
        }
        const size_t c = at(sx, sy);
        if (denRaw > 1e-8) {
            double gVarC = gDen * kEff;
            if (lumaC * lumaC * relEff > epsF) gLumaC += gDen * 2.0 * lumaC * relEff;
            if (varRaw > 0.0) {
                gH[c * 4 + 3] += gVarC;
                gLumaC -= 2.0 * lumaC * gVarC;
            }
        }
        gEC = gEC + V3<double>(0.2126, 0.7152, 0.0722) * gLumaC;
        gH[c * 4] += gEC.x;
        gH[c * 4 + 1] += gEC.y;
        gH[c * 4 + 2] += gEC.z;
    }
}

// Reverse of blend_probe (irradiance part) for one probe: gH (64 x RGBM) of the
// blended history -> gPrev (64 x RGBM, written) and gRays (N x 3, written).
inline void adj_blend_bwd(const Grid& g, const Params& P, const double* rays, const double* Hprev, const double* gH,
                          double* gPrev, double* gRays) {
    const uint32_t N = g.rays;
    std::vector<V3<double>> dirs(N);
    for (uint32_t k = 0; k < N; ++k) dirs[k] = ray_dir<double>(k, N, P.frameJitter);
    std::fill(gPrev, gPrev + 64 * 4, 0.0);
    std::fill(gRays, gRays + (size_t)N * 3, 0.0);
    const V3<double> LW(0.2126, 0.7152, 0.0722);
    for (int lane = 0; lane < 36; ++lane) {
        int lx = lane % OCT_RES + BORDER, ly = lane / OCT_RES + BORDER, local = ly * TILE + lx;
        V3<double> dir = oct_decode((lx - BORDER + 0.5) / OCT_RES, (ly - BORDER + 0.5) / OCT_RES);
        std::vector<double> cw(N);
        V3<double> acc;
        double wsum = 0, lAcc = 0, lAcc2 = 0;
        for (uint32_t k = 0; k < N; ++k) {
            V3<double> r(rays[k * 4], rays[k * 4 + 1], rays[k * 4 + 2]);
            cw[k] = std::pow(std::max(dot(dir, dirs[k]), 0.0), std::max(P.debugCosinePower, 1e-4));
            acc = acc + r * cw[k];
            wsum += cw[k];
            double rl = luma(r);
            lAcc += rl * cw[k];
            lAcc2 += rl * rl * cw[k];
        }
        double wden = std::max(wsum, 1e-4);
        V3<double> meanRad = acc * (1.0 / wden);
        double curL = lAcc / wden, curM2 = lAcc2 / wden;
        const double* p4 = Hprev + (size_t)local * 4;
        V3<double> prev(p4[0], p4[1], p4[2]);
        double prevM2 = p4[3];
        V3<double> gBl(gH[local * 4], gH[local * 4 + 1], gH[local * 4 + 2]);
        double gM2 = gH[local * 4 + 3];
        V3<double> gMean, gPrevV;
        double gCurL = 0, gCurM2 = 0, gPrevM2 = 0;
        if ((prev.x + prev.y + prev.z) < 1e-6) {
            gMean = gBl;
            gCurM2 = gM2;
        } else {
            double prevL = luma(prev);
            double prevVarRaw = prevM2 - prevL * prevL, curVarRaw = curM2 - curL * curL;
            double prevVar = std::max(prevVarRaw, 0.0), curVar = std::max(curVarRaw, 0.0);
            double lumRef = std::max(std::max(curL, prevL), 0.0);
            double varFloor = P.debugTempVarEps + lumRef * lumRef * P.debugTempVarRel;
            double sigma = std::sqrt(prevVar + curVar + varFloor);
            double delta = curL - prevL, absDelta = std::fabs(delta);
            double c0 = P.debugTempChangeSigma0, c1 = std::max(P.tempChangeSigma1, P.debugTempChangeSigma0 + 0.01);
            double s0 = sigma * c0, s1 = sigma * c1, cden = std::max(s1 - s0, 1e-6);
            double x = (absDelta - s0) / cden, changeW = clampv(x, 0.0, 1.0);
            double Hh = P.hysteresis;
            double rawNoiseH = Hh + (1.0 - Hh) * P.debugTempNoiseHBoost;
            double rawChangeH = std::max(Hh - P.tempChangeHDrop, P.debugTempMinChangeH);
            double rawHEff = mixv(rawNoiseH, rawChangeH, changeW), hc = clampv(rawHEff, 1e-6, 1.0);
            double h = std::pow(hc, P.hysteresisExponent);
            double bandIn = prevVar + varFloor, band = std::sqrt(bandIn) * P.tempClampSigma;
            double D = std::max(absDelta, 1e-6), ratio = band / D, cs = std::min(1.0, ratio);
            V3<double> cand = prev + (meanRad - prev) * cs;
            V3<double> gCand = gBl * (1.0 - h);
            gPrevV = gBl * h;
            gCurM2 = gM2 * (1.0 - h);
            gPrevM2 = gM2 * h;
            double gh = dot(gBl, prev - cand) + gM2 * (prevM2 - curM2);
            gMean = gCand * cs;
            gPrevV = gPrevV + gCand * (1.0 - cs);
            double gcs = dot(gCand, meanRad - prev);
            double gAbs = 0, gPrevVar = 0, gCurVar = 0, gVarFloor = 0;
            if (ratio < 1.0) {
                double gBand = gcs / D;
                if (absDelta > 1e-6) gAbs -= gcs * ratio / D;
                if (bandIn > 0.0) {
                    double gIn = gBand * P.tempClampSigma * 0.5 / std::sqrt(bandIn);
                    gPrevVar += gIn;
                    gVarFloor += gIn;
                }
            }
            if (rawHEff > 1e-6 && rawHEff < 1.0) {
                double gRaw = gh * P.hysteresisExponent * std::pow(hc, P.hysteresisExponent - 1.0);
                double gChange = gRaw * (rawChangeH - rawNoiseH);
                if (x > 0.0 && x < 1.0) {
                    gAbs += gChange / cden;
                    double gs0 = -gChange / cden, gs1 = 0.0;
                    if (s1 - s0 > 1e-6) {
                        double gCden = -gChange * x / cden;
                        gs1 += gCden;
                        gs0 -= gCden;
                    }
                    double gSigma = gs0 * c0 + gs1 * c1;
                    if (sigma > 0.0) {
                        double gV = gSigma * 0.5 / sigma;
                        gPrevVar += gV;
                        gCurVar += gV;
                        gVarFloor += gV;
                    }
                }
            }
            double gPrevL = 0.0, gLumRef = gVarFloor * 2.0 * lumRef * P.debugTempVarRel;
            if (lumRef > 0.0) {
                if (curL >= prevL) gCurL += gLumRef;
                else gPrevL += gLumRef;
            }
            double sgn = delta >= 0.0 ? 1.0 : -1.0;
            gCurL += gAbs * sgn;
            gPrevL -= gAbs * sgn;
            if (curVarRaw > 0.0) {
                gCurM2 += gCurVar;
                gCurL -= 2.0 * curL * gCurVar;
            }
            if (prevVarRaw > 0.0) {
                gPrevM2 += gPrevVar;
                gPrevL -= 2.0 * prevL * gPrevVar;
            }
            gPrevV = gPrevV + LW * gPrevL;
        }
        gPrev[local * 4] = gPrevV.x;
        gPrev[local * 4 + 1] = gPrevV.y;
        gPrev[local * 4 + 2] = gPrevV.z;
        gPrev[local * 4 + 3] = gPrevM2;
        for (uint32_t k = 0; k < N; ++k) {
            V3<double> r(rays[k * 4], rays[k * 4 + 1], rays[k * 4 + 2]);
            double a = cw[k] / wden;
            V3<double> gr = gMean * a + LW * (a * (gCurL + 2.0 * luma(r) * gCurM2));
            gRays[k * 3] += gr.x;
            gRays[k * 3 + 1] += gr.y;
            gRays[k * 3 + 2] += gr.z;
        }
    }
}

// Reverse pass. grad = [albedo mc x 3 | emissive mc x 3 | light scale lc].
inline void adj_backward(const AdjProblem& A, const AdjTape& T, const double* target, double* grad) {
    const Grid& g = A.g;
    const uint32_t probes = g.probeTotal(), N = g.rays, mc = A.materialCount, lc = A.lightCount;
    const size_t texels = (size_t)g.atlasW() * g.atlasH(), nParam = 6 * (size_t)mc + lc, hsz = (size_t)probes * 256;
    const int nt = std::max(1, A.threads);
    std::vector<double> gE(T.E.size());
    for (size_t i = 0; i < gE.size(); ++i) gE[i] = 2.0 * (T.E[i] - target[i]);
    std::vector<double> gHnext(hsz, 0.0), gHprev(hsz), gAnext, rays, gR((size_t)probes * N * 3);
    std::vector<std::vector<double>> gParamT(nt, std::vector<double>(nParam, 0.0));
    std::vector<std::vector<double>> gAT(nt);
    for (int s = (int)A.solves - 1; s >= 0; --s) {
        const bool last = s + 1 == (int)A.solves;
        const std::vector<double>& H1 = T.hist[s + 1];
        adj_parallel(probes, nt, [&](size_t p, int) {
            double gEp[36 * 3];
            for (int i = 0; i < 108; ++i) gEp[i] = last ? gE[p * 108 + i] : 0.0;
            if (!gAnext.empty()) {
                uint32_t col = (uint32_t)p % g.res[0];
                uint32_t row = ((uint32_t)p / (g.res[0] * g.res[1])) * g.res[1] + ((uint32_t)p / g.res[0]) % g.res[1];
                for (int lane = 0; lane < TILE * TILE; ++lane) {
                    size_t t = (size_t)(row * TILE + lane / TILE) * g.atlasW() + col * TILE + lane % TILE;
                    int src = gutter_source_lane(lane);
                    for (int c = 0; c < 3; ++c) gEp[src * 3 + c] += gAnext[t * 3 + c];
                }
            }
            adj_upload_bwd(A.P, H1.data() + p * 256, gEp, gHnext.data() + p * 256);
        });
        adj_rays(A, T.atlas[s].data(), rays);
        adj_parallel(probes, nt, [&](size_t p, int) {
            adj_blend_bwd(g, A.P, rays.data() + p * N * 4, T.hist[s].data() + p * 256, gHnext.data() + p * 256,
                          gHprev.data() + p * 256, gR.data() + p * N * 3);
        });
        for (auto& a : gAT) a.assign(texels * 3, 0.0);
        Replay rp{A.tri, A.inst, A.blocked};
        adj_parallel((size_t)probes * N, nt, [&](size_t i, int th) {
            V3<double> gr(gR[i * 3], gR[i * 3 + 1], gR[i * 3 + 2]);
            if (A.tri[i] < 0 || (gr.x == 0.0 && gr.y == 0.0 && gr.z == 0.0)) return;
            Tracer<double> tc = adj_tracer(A, T.atlas[s].data());
            typename Tracer<double>::ShadeRecord rec;
            tc.rec = &rec;
            RayOut<double> o;
            tc.trace((uint32_t)(i / N), (uint32_t)(i % N), 0, o, &rp, i);
            if (!rec.hit) return;
            double* gp = gParamT[th].data();
            const uint32_t m = rec.m;
            V3<double> gEm = gr * A.P.debugEmissiveScale;
            V3<double> gkd;
            for (uint32_t j = 0; j < rec.nLights; ++j) {
                gp[6 * (size_t)mc + rec.li[j]] += dot(gr, mulv(rec.X[j], rec.kd));
                gkd = gkd + mulv(gr, rec.X[j]);
            }
            const double C = A.P.radianceClamp, bs = A.P.debugBounceScale;
            const double bl = luma(rec.bounce), rden = std::max(std::max(C, bl), 1e-6);
            V3<double> gB;
            if (bl > C && bl > 1e-6) {
                double k1 = C * bs / rden;
                gB = gr * k1 - V3<double>(0.2126, 0.7152, 0.0722) * (dot(gr, rec.bounce) * k1 / rden);
            } else {
                gB = gr * (C / rden * bs);
            }
            V3<double> gS = mulv(gB, rec.kd) * (1.0 / PI);
            gkd = gkd + mulv(gB, rec.smp) * (1.0 / PI);
            size_t idx[32];
            double wt[32];
            adj_atlas_taps(g, rec.hitPos, rec.ng, idx, wt);
            double* ga = gAT[th].data();
            for (int q = 0; q < 32; ++q) {
                ga[idx[q] * 3] += gS.x * wt[q];
                ga[idx[q] * 3 + 1] += gS.y * wt[q];
                ga[idx[q] * 3 + 2] += gS.z * wt[q];
            }
            const double kdc[3] = {rec.kdr.x, rec.kdr.y, rec.kdr.z}, gkc[3] = {gkd.x, gkd.y, gkd.z};
            const double gec[3] = {gEm.x, gEm.y, gEm.z};
            for (int c = 0; c < 3; ++c) {
                if (kdc[c] > 0.0 && kdc[c] < 0.95) gp[3 * m + c] += gkc[c] * rec.kdScale;
                gp[3 * ((size_t)mc + m) + c] += gec[c];
            }
        });
        gAnext.assign(texels * 3, 0.0);
        for (auto& a : gAT)
            for (size_t i = 0; i < a.size(); ++i) gAnext[i] += a[i];
        gHnext.swap(gHprev);
    }
    std::fill(grad, grad + nParam, 0.0);
    for (auto& gp : gParamT)
        for (size_t i = 0; i < nParam; ++i) grad[i] += gp[i];
}

}  // namespace orc
