// orc_api.cpp — extern "C" surface of the oracle for the tests (ctypes) and
// bench.py's CPU baseline. TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
#include "orc_probes.hpp"
#include "orc_scene.hpp"
#include "orc_bvh.hpp"
#include "orc_gather.hpp"

#include <atomic>
#include <thread>

using namespace orc;


struct OrcScene {
    const uint32_t* nodes; uint32_t nodeCount;
    const uint32_t* triIndex; uint32_t triCount;
    const float* vertexData; uint32_t vertexCount;
    const uint32_t* triMaterial;
    const float* materials; uint32_t materialsLen;
    uint32_t instBase, instCount, tlasBase, tlasNodeCount;
};
struct OrcLights {
    const float* data; uint32_t dataLen; uint32_t lightCount; int32_t clustered;
    uint32_t emitterBase, emitterCount;
};
struct OrcGrid { double gridMin[3], gridSize[3]; uint32_t res[3]; uint32_t rays; double maxDist, cellMin; };

// Optional per-ray outputs / replay inputs of a solve. Any pointer may be null.
struct OrcSolveIO {
    void* rayOut;             // R[updated*rays*4]: rgb + hitT
    int32_t* hitTri; int32_t* hitInst;
    void* secondT;            // R per ray
    uint64_t* tested; uint64_t* blocked;
    const int32_t* replayTri; const int32_t* replayInst; const uint64_t* replayBlocked;
    const void* rayIn;        // R rays to blend instead of tracing (replay of the blend alone)
    void* preRound;           // R[probeTotal*36*3]: unrounded upload RGB
    uint64_t* counters;       // [tlasNodes, instances, blasNodes, triTests] (primary + shadow)
    int32_t* hitFacing;       // per ray: 1 front, 0 back, -1 miss
    void* emitterVis;         // R[probeTotal*16]: emitter visibility history (in/out), or null
    const void* emitterVisReplay;  // R[probeTotal*16]: the GPU's history after the solve, taken for the
                                   // updated probes before the blend (replay), or null
    void* emitterSampleOut;   // R[updated*16]: this solve's own visibility samples, or null
    // reflection lobes (tier 0 off, 1 rough, 2 high, 3 ultra); the buffers are
    // in/out and sized for the tier (glossy tile = 10 / 18 texels a side)
    uint32_t reflectTier, glossyPhase;
    void* roughSpec;          // R[probeTotal*64*4]
    uint16_t* roughAtlas;     // RGBA16F, atlasW*atlasH*4
    void* glossyNum;          // R[probeTotal*tile^2*4]
    void* glossyDen;          // R[probeTotal*tile^2]
    uint16_t* glossyAtlas;    // RGBA16F, (tilesX*tile)*(tilesY*tile)*4
};


static Scene to_scene(const OrcScene* s) {
    Scene sc;
    sc.nodes = s->nodes; sc.nodeCount = s->nodeCount; sc.triIndex = s->triIndex; sc.triCount = s->triCount;
    sc.vertexData = s->vertexData; sc.vertexCount = s->vertexCount; sc.triMaterial = s->triMaterial;
    sc.materials = s->materials; sc.materialsLen = s->materialsLen; sc.instBase = s->instBase;
    sc.instCount = s->instCount; sc.tlasBase = s->tlasBase; sc.tlasNodeCount = s->tlasNodeCount;
    return sc;
}
static Grid to_grid(const OrcGrid* g) {
    Grid o;
    for (int i = 0; i < 3; ++i) { o.gridMin[i] = g->gridMin[i]; o.gridSize[i] = g->gridSize[i]; o.res[i] = g->res[i]; }
    o.rays = g->rays; o.maxDist = g->maxDist; o.cellMin = g->cellMin;
    return o;
}

template <class F> static void parallel_for(size_t n, int threads, F&& f) {
    if (threads <= 1 || n < 64) { for (size_t i = 0; i < n; ++i) f(i, 0); return; }
    std::atomic<size_t> next{0};
    std::vector<std::thread> ts;
    const size_t chunk = 64;
    for (int t = 0; t < threads; ++t)
        ts.emplace_back([&, t] {
            for (;;) {
                size_t b = next.fetch_add(chunk);
                if (b >= n) break;
                size_t e = std::min(n, b + chunk);
                for (size_t i = b; i < e; ++i) f(i, t);
            }
        });
    for (auto& th : ts) th.join();
}

extern "C" {

int orc_version(void) { return 1; }

// -------------------------------------------------------------- traversal
void orc_closest(const OrcScene* s, const float* ro, const float* rd, uint32_t n, int32_t track2, int32_t brute,
                 double* tOut, int32_t* triOut, int32_t* instOut, double* secondOut, int32_t threads) {
    Scene sc = to_scene(s);
    parallel_for(n, threads, [&](size_t i, int) {
        Traverser<double> tr(sc);
        tr.track2 = track2 != 0;
        V3<double> o(ro[i * 3], ro[i * 3 + 1], ro[i * 3 + 2]), d(rd[i * 3], rd[i * 3 + 1], rd[i * 3 + 2]);
        double t, t2 = T_MAX;
        int tri, inst;
        if (brute) tr.brute_closest(o, d, t, tri, inst);
        else tr.closest(o, d, t, tri, inst, t2);
        tOut[i] = t; triOut[i] = tri; instOut[i] = inst;
        if (secondOut) secondOut[i] = t2;
    });
}

void orc_any(const OrcScene* s, const float* ro, const float* rd, const float* maxDist, uint32_t n, uint8_t* blocked,
             int32_t threads) {
    Scene sc = to_scene(s);
    parallel_for(n, threads, [&](size_t i, int) {
        Traverser<double> tr(sc);
        V3<double> o(ro[i * 3], ro[i * 3 + 1], ro[i * 3 + 2]), d(rd[i * 3], rd[i * 3 + 1], rd[i * 3 + 2]);
        blocked[i] = tr.any(o, d, (double)maxDist[i]) ? 1 : 0;
    });
}

}  // extern "C"

// ------------------------------------------------ hit-ID disagreement proof
// One (triangle, instance slot) pair evaluated on a world ray in FP64 with the
// reference's Möller–Trumbore (spectral_traverse.js:393-409) and its closest-hit
// acceptance (side, alpha/const-alpha flags, 193-220), plus a first-order bound
// on how far an FP32 evaluation of the same test can move u, v and t. The bound
// sums the magnitudes of the terms each FP32 operation rounds: the world-to-local
// transform (inverse rows · origin + translation), the edge vectors, the two
// cross products and the three dot products, each term rounded at most a few
// times with unit roundoff 2^-24; a factor 16 covers the operation count.
struct PairEval {
    bool valid = false;    // tri >= 0 and the slot is live
    bool accepted = false; // MT passes and the pair is accepted as a closest hit
    bool rejectedByBary = false;  // only u/v (edge) conditions reject it
    double t = 0, u = 0, v = 0, margin = 0;  // margin = min(u, v, 1-u-v)
    double tauBary = 0, tauT = 0;
};

static PairEval eval_pair(const Traverser<double>& tr, const Scene& s, int tri, int inst, V3<double> wro, V3<double> wrd) {
    PairEval e;
    if (tri < 0 || inst < 0 || (uint32_t)tri >= s.triCount || (uint32_t)inst >= s.instCount) return e;
    e.valid = true;
    V3<double> ro = tr.inst_inv_point((uint32_t)inst, wro), rd = tr.inst_inv_dir((uint32_t)inst, wrd);
    double dSign = tr.inst_f((uint32_t)inst, 14);
    double Mn = 0, Wn = 0;
    for (int r = 0; r < 3; ++r) {
        Mn += length(tr.inst_row((uint32_t)inst, r));
        Wn += std::fabs(tr.inst_f((uint32_t)inst, r * 4 + 3));
    }
    V3<double> p0 = tr.fetch_vert(tr.tri_vert(tri, 0)), p1 = tr.fetch_vert(tr.tri_vert(tri, 1)),
               p2 = tr.fetch_vert(tr.tri_vert(tri, 2));
    V3<double> e1 = p1 - p0, e2 = p2 - p0, pv = cross(rd, e2), tv = ro - p0, qv = cross(tv, e1);
    double det = dot(e1, pv);
    if (!(std::fabs(det) > 1e-12)) return e;
    double inv = 1.0 / det;
    e.u = dot(tv, pv) * inv;
    e.v = dot(rd, qv) * inv;
    e.t = dot(e2, qv) * inv;
    e.margin = std::min(std::min(e.u, e.v), 1.0 - e.u - e.v);
    const double eps = 16.0 * std::ldexp(1.0, -24);
    // magnitudes entering the FP32 evaluation
    double S = Mn * length(wro) + Wn + length(ro) + length(p0) + length(p1) + length(p2);  // origin side
    double D = Mn * length(wrd) + length(rd);                                                // direction side
    double E1 = length(e1) + length(p0) + length(p1), E2 = length(e2) + length(p0) + length(p2);
    double dDet = eps * (E1 * D * E2);
    double dNu = eps * (S * length(pv) + length(tv) * D * E2);
    double dNv = eps * (D * S * E1 + length(qv) * D);
    double dNt = eps * (E2 * length(qv) + E2 * S * E1);
    double ad = std::fabs(det);
    double du = (dNu + std::fabs(e.u) * dDet) / ad, dv = (dNv + std::fabs(e.v) * dDet) / ad;
    e.tauBary = du + dv;
    e.tauT = (dNt + std::fabs(e.t) * dDet) / ad;
    bool baryOk = e.u >= 0.0 && e.u <= 1.0 && e.v >= 0.0 && e.u + e.v <= 1.0;
    uint32_t m = s.triMaterial[tri];
    uint32_t fl = tr.flags(m);
    bool acc = tr.side_accepts(m, det * dSign) && ((fl & 1u) ? tr.alpha_accepts(m) : (fl & 2u) != 0);
    bool active = tr.inst_f((uint32_t)inst, 15) > 0.5;
    bool tOk = e.t > RAY_EPS;
    e.accepted = active && acc && tOk && baryOk;
    e.rejectedByBary = active && acc && tOk && !baryOk;
    return e;
}

extern "C" {

// World-space probe rays of a solve in FP64: ray i = (slot i / rays, k i % rays),
// probe (probeOffset + slot) mod probeTotal (gi_probes.js:1977-1987).
void orc_probe_rays(const OrcGrid* gp, double jitter, uint32_t probeOffset, uint32_t updated, double* roOut,
                    double* rdOut) {
    Grid g = to_grid(gp);
    const uint32_t N = g.rays, total = g.probeTotal();
    for (size_t i = 0; i < (size_t)updated * N; ++i) {
        uint32_t slot = (uint32_t)(i / N), k = (uint32_t)(i % N);
        V3<double> o = probe_world_pos<double>(g, (probeOffset + slot) % total);
        V3<double> d = ray_dir<double>(k, N, jitter);
        roOut[i * 3] = o.x; roOut[i * 3 + 1] = o.y; roOut[i * 3 + 2] = o.z;
        rdOut[i * 3] = d.x; rdOut[i * 3 + 1] = d.y; rdOut[i * 3 + 2] = d.z;
    }
}

// FP64 t of the pair (tri[i], inst[i]) on ray i (-1 where there is no pair or
// the Möller–Trumbore determinant vanishes): the exact ray parameter of a
// reported hit, for checking the reported t on the ray that was traced.
void orc_pair_t(const OrcScene* s, const double* ro, const double* rd, uint32_t n, const int32_t* tri,
                const int32_t* inst, double* tOut, int32_t threads) {
    Scene sc = to_scene(s);
    parallel_for(n, threads, [&](size_t i, int) {
        Traverser<double> tr(sc);
        V3<double> o(ro[i * 3], ro[i * 3 + 1], ro[i * 3 + 2]), d(rd[i * 3], rd[i * 3 + 1], rd[i * 3 + 2]);
        PairEval e = eval_pair(tr, sc, tri[i], inst[i], o, d);
        tOut[i] = e.valid && e.t != 0.0 ? e.t : -1.0;
    });
}

// Classifies every ray whose GPU closest hit (gTri, gInst) differs from the FP64
// oracle's (oTri, oInst, oT). Codes:
//   0 same pair;
//   1 near-tie: both pairs accepted in FP64, their t within 1e-6 relative;
//   2 the GPU's pair is an edge graze: FP64 rejects it only by its barycentric
//     bounds, by less than the FP32 bound, and it lies no farther than the
//     oracle's hit (or the oracle missed);
//   3 the oracle's pair is an edge graze: accepted in FP64 within the FP32 bound
//     of an edge, and the GPU's hit (if any) is an accepted pair no nearer;
//   4 t-order within FP32 error: both accepted, |t_g - t_o| within the FP32 t
//     bounds of the two pairs;
//   5 unexplained.
// gTOut receives the FP64 t of the GPU's pair (or -1).
void orc_explain_hits(const OrcScene* s, const double* ro, const double* rd, uint32_t n, const int32_t* gTri,
                      const int32_t* gInst, const int32_t* oTri, const int32_t* oInst, const double* oT,
                      int32_t* codeOut, double* gTOut, int32_t threads) {
    Scene sc = to_scene(s);
    parallel_for(n, threads, [&](size_t i, int) {
        gTOut[i] = -1.0;
        if (gTri[i] == oTri[i] && (gTri[i] < 0 || gInst[i] == oInst[i])) { codeOut[i] = 0; return; }
        Traverser<double> tr(sc);
        V3<double> o(ro[i * 3], ro[i * 3 + 1], ro[i * 3 + 2]), d(rd[i * 3], rd[i * 3 + 1], rd[i * 3 + 2]);
        PairEval g = eval_pair(tr, sc, gTri[i], gInst[i], o, d);
        PairEval r = eval_pair(tr, sc, oTri[i], oInst[i], o, d);
        if (g.valid) gTOut[i] = g.t;
        const double tO = oTri[i] >= 0 ? oT[i] : INFINITY;
        int code = 5;
        if (g.accepted && r.accepted && std::fabs(g.t - r.t) <= 1e-6 * std::fabs(r.t)) code = 1;
        else if (g.valid && g.rejectedByBary && g.margin >= -g.tauBary && g.t <= tO * (1 + 1e-6)) code = 2;
        else if (r.valid && r.accepted && r.margin <= r.tauBary && (!g.valid || (g.accepted && g.t >= tO * (1 - 1e-6)) ||
                 (g.rejectedByBary && g.margin >= -g.tauBary)))
            code = 3;
        else if (g.accepted && r.accepted && std::fabs(g.t - r.t) <= g.tauT + r.tauT) code = 4;
        codeOut[i] = code;
    });
}

}  // extern "C"

// ------------------------------------------------------------------ solve
template <class R>
static int solve_impl(const OrcScene* s, const OrcLights* l, const OrcGrid* gp, const OrcGrid* g0p, const double* params,
                      uint32_t probeOffset, uint32_t updated, R* irr, R* depth, uint16_t* atlas, uint16_t* depthAtlas,
                      OrcSolveIO* io, int32_t threads) {
    Scene sc = to_scene(s);
    Grid g = to_grid(gp), g0 = to_grid(g0p ? g0p : gp);
    Params P;
    std::memcpy(&P, params, sizeof(Params));
    Lights L;
    L.data = l->data; L.dataLen = l->dataLen; L.lightCount = l->lightCount; L.clustered = l->clustered;
    L.emitterBase = l->emitterBase; L.emitterCount = l->emitterCount;
    const uint32_t N = g.rays, total = g.probeTotal();
    if (updated > total) updated = total;
    const size_t nr = (size_t)updated * N;
    std::vector<R> rays;
    const R* rayBuf;
    Replay rp{nullptr, nullptr, nullptr};
    if (io && io->replayTri) { rp.tri = io->replayTri; rp.inst = io->replayInst; rp.blocked = io->replayBlocked; }
    if (io && io->rayIn) {
        rayBuf = static_cast<const R*>(io->rayIn);
    } else {
        rays.assign(nr * 4, R(0));
        int nt = std::max(1, threads);
        std::vector<Counters> cnts(nt);
        parallel_for(nr, nt, [&](size_t i, int t) {
            Tracer<R> tc(sc, L, g, g0, P, atlas);
            tc.roughEncode = io && io->reflectTier >= 1;
            if (io && io->counters) tc.tr.cnt = &cnts[t];
            RayOut<R> o;
            uint32_t slot = (uint32_t)(i / N), k = (uint32_t)(i % N);
            tc.trace(slot, k, probeOffset, o, rp.tri ? &rp : nullptr, i);
            rays[i * 4] = o.rgb[0]; rays[i * 4 + 1] = o.rgb[1]; rays[i * 4 + 2] = o.rgb[2]; rays[i * 4 + 3] = o.hitT;
            if (io) {
                if (io->hitTri) io->hitTri[i] = o.tri;
                if (io->hitInst) io->hitInst[i] = o.inst;
                if (io->secondT) static_cast<R*>(io->secondT)[i] = o.secondT;
                if (io->tested) io->tested[i] = o.tested;
                if (io->blocked) io->blocked[i] = o.blocked;
                if (io->hitFacing) io->hitFacing[i] = o.tri >= 0 ? o.facing : -1;
            }
        });
        if (io && io->counters) {
            Counters c;
            for (auto& x : cnts) c.add(x);
            io->counters[0] = c.tlasNodes; io->counters[1] = c.instances; io->counters[2] = c.blasNodes; io->counters[3] = c.triTests;
        }
        rayBuf = rays.data();
        if (io && io->rayOut) std::memcpy(io->rayOut, rays.data(), nr * 4 * sizeof(R));
    }
    R* pre = io ? static_cast<R*>(io->preRound) : nullptr;
    // emitterVisKernel (gi_probes.js:2216-2260), after the trace and before the blend
    R* evis = io ? static_cast<R*>(io->emitterVis) : nullptr;
    if (evis && L.emitterCount) {
        const uint32_t EC = GI_EMITTER_INJECT_CAP;
        R* sampleOut = static_cast<R*>(io->emitterSampleOut);
        parallel_for((size_t)updated * EC, std::max(1, threads), [&](size_t i, int) {
            uint32_t slot = (uint32_t)(i / EC), e = (uint32_t)(i % EC);
            if (e >= L.emitterCount) return;
            uint32_t p = (uint32_t)((probeOffset + slot) % total);
            R smp = emitter_sample<R>(sc, L, g, P, p, e);
            if (sampleOut) sampleOut[i] = smp;
            R& v = evis[(size_t)p * EC + e];
            v = smp * (R(1) - R(GI_EMITTER_VIS_RETENTION)) + v * R(GI_EMITTER_VIS_RETENTION);
        });
        if (io->emitterVisReplay) {
            const R* rv = static_cast<const R*>(io->emitterVisReplay);
            for (uint32_t slot = 0; slot < updated; ++slot) {
                uint32_t p = (uint32_t)((probeOffset + slot) % total);
                for (uint32_t e = 0; e < EC; ++e) evis[(size_t)p * EC + e] = rv[(size_t)p * EC + e];
            }
        }
    }
    EmitterInject<R> inj;
    inj.L = &L;
    inj.vis = evis;
    Reflect<R> rf;
    if (io && io->reflectTier) {
        rf.tier = io->reflectTier;
        rf.roughSpec = static_cast<R*>(io->roughSpec);
        rf.roughAtlas = io->roughAtlas;
        rf.glossyNum = static_cast<R*>(io->glossyNum);
        rf.glossyDen = static_cast<R*>(io->glossyDen);
        rf.glossyAtlas = io->glossyAtlas;
        rf.glossyPhase = io->glossyPhase;
        if (!rf.roughSpec || !rf.roughAtlas) return 2;
        if (rf.tier >= 2 && (!rf.glossyNum || !rf.glossyDen || !rf.glossyAtlas)) return 2;
    }
    Reflect<R>* rfp = rf.tier ? &rf : nullptr;
    parallel_for(updated, std::max(1, threads), [&](size_t slot, int) {
        uint32_t p = (uint32_t)((probeOffset + slot) % total);
        blend_probe<R>(g, P, rayBuf + slot * N * 4, p, irr, depth, evis ? &inj : nullptr, rfp);
    });
    // glossyKernel, then the upload (gi_probes.js:3829-3836)
    if (rf.tier >= 2)
        parallel_for(updated, std::max(1, threads), [&](size_t slot, int) {
            uint32_t p = (uint32_t)((probeOffset + slot) % total);
            glossy_probe<R>(g, P, rayBuf + slot * N * 4, p, rf, evis ? &inj : nullptr);
        });
    parallel_for(updated, std::max(1, threads), [&](size_t slot, int) {
        uint32_t p = (uint32_t)((probeOffset + slot) % total);
        upload_probe<R>(g, P, p, irr, depth, atlas, depthAtlas, pre, rfp);
    });
    return 0;
}

extern "C" {

int orc_solve_f64(const OrcScene* s, const OrcLights* l, const OrcGrid* g, const OrcGrid* g0, const double* params,
                  uint32_t probeOffset, uint32_t updated, double* irr, double* depth, uint16_t* atlas,
                  uint16_t* depthAtlas, OrcSolveIO* io, int32_t threads) {
    return solve_impl<double>(s, l, g, g0, params, probeOffset, updated, irr, depth, atlas, depthAtlas, io, threads);
}
int orc_solve_f32(const OrcScene* s, const OrcLights* l, const OrcGrid* g, const OrcGrid* g0, const double* params,
                  uint32_t probeOffset, uint32_t updated, float* irr, float* depth, uint16_t* atlas,
                  uint16_t* depthAtlas, OrcSolveIO* io, int32_t threads) {
    return solve_impl<float>(s, l, g, g0, params, probeOffset, updated, irr, depth, atlas, depthAtlas, io, threads);
}

uint32_t orc_params_size(void) { return (uint32_t)(sizeof(Params) / sizeof(double)); }

// Receiver gather (orc_gather.hpp) of n surface points, FP64. pos/nvis/ndir are
// 4 floats per point (xyz used); out is 3 doubles per point; near (may be null)
// receives each point's distance to a discontinuity of the gather.
void orc_gather(const OrcGrid* g0, const OrcGrid* g1, const uint16_t* atlas0, const uint16_t* depth0,
                const uint16_t* atlas1, const uint16_t* depth1, const double* params, const float* pos4,
                const float* nvis4, const float* ndir4, uint32_t n, double* out3, double* near, int32_t threads) {
    Grid G0 = to_grid(g0), G1;
    if (g1) G1 = to_grid(g1);
    GatherParams prm;
    std::memcpy(&prm, params, sizeof prm);
    GatherCascade C[2];
    C[0].g = &G0; C[0].atlas = atlas0; C[0].depth = depth0;
    if (g1) { C[1].g = &G1; C[1].atlas = atlas1; C[1].depth = depth1; }
    parallel_for(n, threads, [&](size_t i, int) {
        V3<double> p(pos4[i * 4], pos4[i * 4 + 1], pos4[i * 4 + 2]);
        V3<double> a(nvis4[i * 4], nvis4[i * 4 + 1], nvis4[i * 4 + 2]);
        V3<double> b(ndir4[i * 4], ndir4[i * 4 + 1], ndir4[i * 4 + 2]);
        double nr = INFINITY;
        V3<double> e = gather_point<double>(C, prm, p, a, b, nr);
        out3[i * 3] = e.x; out3[i * 3 + 1] = e.y; out3[i * 3 + 2] = e.z;
        if (near) near[i] = nr;
    });
}
uint32_t orc_gather_params_size(void) { return (uint32_t)(sizeof(GatherParams) / sizeof(double)); }

// The reflection atlases of one cascade for the combined receiver: rough in the
// irradiance layout; glossy (null below tier high) with its tile geometry.
struct OrcReflectAtlas {
    const uint16_t* rough; const uint16_t* glossy;
    uint32_t glossyOct, glossyTile, glossyTilesX, glossyW, glossyH;
};

// Combined receiver (orc_gather.hpp combined_point) of n points, FP64.
// rdir4: reflection direction xyz + roughness w; outIrr 3 doubles and outRefl
// 4 doubles per point; near (may be null) as orc_gather.
void orc_gather_combined(const OrcGrid* g0, const OrcGrid* g1, const uint16_t* atlas0, const uint16_t* depth0,
                         const uint16_t* atlas1, const uint16_t* depth1, const OrcReflectAtlas* r0,
                         const OrcReflectAtlas* r1, const double* params, const float* pos4, const float* nvis4,
                         const float* ndir4, const float* rdir4, uint32_t n, double* outIrr, double* outRefl,
                         double* near, int32_t threads) {
    Grid G0 = to_grid(g0), G1;
    if (g1) G1 = to_grid(g1);
    GatherParams prm;
    std::memcpy(&prm, params, sizeof prm);
    GatherCascade C[2];
    C[0].g = &G0; C[0].atlas = atlas0; C[0].depth = depth0;
    if (g1) { C[1].g = &G1; C[1].atlas = atlas1; C[1].depth = depth1; }
    const OrcReflectAtlas* rs[2] = {r0, r1};
    for (int c = 0; c < 2; ++c) {
        if (!rs[c]) continue;
        C[c].rough = rs[c]->rough; C[c].glossy = rs[c]->glossy;
        C[c].glossyOct = rs[c]->glossyOct; C[c].glossyTile = rs[c]->glossyTile;
        C[c].glossyTilesX = rs[c]->glossyTilesX; C[c].glossyW = rs[c]->glossyW; C[c].glossyH = rs[c]->glossyH;
    }
    parallel_for(n, threads, [&](size_t i, int) {
        V3<double> p(pos4[i * 4], pos4[i * 4 + 1], pos4[i * 4 + 2]);
        V3<double> a(nvis4[i * 4], nvis4[i * 4 + 1], nvis4[i * 4 + 2]);
        V3<double> b(ndir4[i * 4], ndir4[i * 4 + 1], ndir4[i * 4 + 2]);
        V3<double> r(rdir4[i * 4], rdir4[i * 4 + 1], rdir4[i * 4 + 2]);
        double nr = INFINITY;
        V3<double> e;
        combined_point<double>(C, prm, p, a, b, r, (double)rdir4[i * 4 + 3], nr, e, outRefl + i * 4);
        outIrr[i * 3] = e.x; outIrr[i * 3 + 1] = e.y; outIrr[i * 3 + 2] = e.z;
        if (near) near[i] = nr;
    });
}

// ------------------------------------------------------------ light grid
void orc_light_grid(const OrcGrid* g0, const float* lights, uint32_t lightCount, float* out, int32_t fp32) {
    Grid g = to_grid(g0);
    if (fp32) light_grid<float>(g, lights, lightCount, out);
    else light_grid<double>(g, lights, lightCount, out);
}

// ------------------------------------------------------------ small KATs
void orc_oct_encode(const double* n, double* uv) { oct_encode(V3<double>(n[0], n[1], n[2]), uv[0], uv[1]); }
void orc_oct_decode(const double* uv, double* n) {
    V3<double> d = oct_decode(uv[0], uv[1]);
    n[0] = d.x; n[1] = d.y; n[2] = d.z;
}
uint16_t orc_to_half(double v) { return to_half(v); }
double orc_from_half(uint16_t h) { return from_half(h); }
void orc_ray_dir(uint32_t k, uint32_t rays, double jitter, double* out) {
    V3<double> d = ray_dir<double>(k, rays, jitter);
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}
void orc_probe_world_pos(const OrcGrid* g, uint32_t p, double* out) {
    Grid gg = to_grid(g);
    V3<double> d = probe_world_pos<double>(gg, p);
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}
double orc_hysteresis_exponent(double dtMs, int32_t normalize) { return hysteresis_exponent_for_interval(dtMs, normalize != 0); }
void orc_grid_resolution(const double* size, int32_t target, uint32_t* out) { compute_grid_resolution(size, target, out); }
int32_t orc_gutter_source_lane(int32_t lane) { return gutter_source_lane(lane); }
void orc_sample_atlas(const OrcGrid* g, const uint16_t* atlas, const double* P, const double* N, double* out) {
    Grid gg = to_grid(g);
    V3<double> r = sample_atlas<double>(gg, atlas, V3<double>(P[0], P[1], P[2]), V3<double>(N[0], N[1], N[2]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// ------------------------------------------------------- refit and TLAS
int32_t orc_refit_blas(uint32_t* nodes, uint64_t nodesLen, const uint32_t* triIndex, uint64_t triIndexLen,
                       const float* vertexData, uint64_t vdLen, int64_t root, int64_t end) {
    return refit_blas(nodes, nodesLen, triIndex, triIndexLen, vertexData, vdLen, root, end) ? 1 : 0;
}
int32_t orc_refit_tlas_range(float* nodes, uint64_t nodesLen, const float* ib, uint64_t ibLen, int64_t root, int64_t end) {
    return refit_tlas_range(nodes, nodesLen, ib, ibLen, root, end) ? 1 : 0;
}
int32_t orc_refit_tlas_dirty(float* nodes, uint64_t nodesLen, const float* ib, uint64_t ibLen, int64_t end,
                             const uint32_t* dirty, uint64_t nDirty, uint32_t* touchedOut, uint32_t* touchedCount) {
    std::vector<uint32_t> t;
    if (!refit_tlas_dirty(nodes, nodesLen, ib, ibLen, end, dirty, nDirty, t)) return 0;
    for (size_t i = 0; i < t.size(); ++i) touchedOut[i] = t[i];
    *touchedCount = (uint32_t)t.size();
    return 1;
}
// MeshBVH build + flattenBVHRoot of one mesh (orc_bvh.hpp). index3 is permuted
// in place into BVH order; orderOut[i] = source triangle at position i.
uint32_t orc_build_blas(const float* pos3, uint32_t vertCount, uint32_t* index3, uint32_t triCount, uint32_t leafSize,
                        uint32_t* nodesOut, uint64_t nodesCap, uint32_t* orderOut) {
    std::vector<uint32_t> nodes, order;
    uint32_t n = build_mesh_bvh(pos3, vertCount, index3, triCount, leafSize, nodes, order);
    if (!n || n > nodesCap) return 0;
    std::memcpy(nodesOut, nodes.data(), (size_t)n * 32);
    std::memcpy(orderOut, order.data(), (size_t)triCount * 4);
    return n;
}
// aabbs9: per instance min xyz, max xyz, centroid xyz (FP64)
uint32_t orc_build_tlas(const double* aabbs9, uint32_t n, float* nodes12Out, uint32_t* orderOut, double* bounds64Out) {
    std::vector<Aabb> a(n);
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            a[i].mn[k] = aabbs9[i * 9 + k]; a[i].mx[k] = aabbs9[i * 9 + 3 + k]; a[i].c[k] = aabbs9[i * 9 + 6 + k];
        }
    std::vector<TlasRec> recs;
    std::vector<uint32_t> order;
    build_tlas(a, recs, order);
    for (size_t i = 0; i < recs.size(); ++i) {
        float* o = nodes12Out + i * 12;
        for (int k = 0; k < 6; ++k) o[k] = (float)recs[i].bx[k];
        o[6] = (float)recs[i].miss;
        o[7] = recs[i].leaf ? (float)recs[i].off : 0.0f;
        o[8] = recs[i].leaf ? (float)recs[i].cnt : 0.0f;
        o[9] = o[10] = o[11] = 0.0f;
        if (bounds64Out) for (int k = 0; k < 6; ++k) bounds64Out[i * 6 + k] = recs[i].bx[k];
    }
    for (uint32_t i = 0; i < n; ++i) orderOut[i] = order[i];
    return (uint32_t)recs.size();
}
// computeDynamic per source instance: world16 column-major FP64, local bounds f32.
void orc_compute_instances(const double* world16, const uint8_t* active, const float* lbounds6, uint32_t n,
                           float* invRows12, float* detSign, double* aabbs9) {
    for (uint32_t i = 0; i < n; ++i) {
        Aabb b;
        compute_instance(world16 + (size_t)i * 16, active[i] != 0, lbounds6 + (size_t)i * 6, invRows12 + (size_t)i * 12,
                         detSign[i], b);
        for (int k = 0; k < 3; ++k) {
            aabbs9[i * 9 + k] = b.mn[k]; aabbs9[i * 9 + 3 + k] = b.mx[k]; aabbs9[i * 9 + 6 + k] = b.c[k];
        }
    }
}

}  // extern "C"

// ------------------------------------------------------------- adjoint
#include "orc_adjoint.hpp"

extern "C" {

// Differentiable solve sequence in FP64 (orc_adjoint.hpp). Replay records are
// per ray of one solve (probe-major, probe index = slot) and serve every solve.
// Parameters: albedo / emissive (materialCount x 3), lightScale (lightCount).
// Outputs (any may be null): loss (needs target), E (probes x 36 x 3), grad
// ([albedo | emissive | light scale], needs target).
int orc_adjoint(const OrcScene* s, const OrcLights* l, const OrcGrid* g, const double* params, const int32_t* tri,
                const int32_t* inst, const uint64_t* blocked, uint32_t solves, int32_t roundAtlas,
                const double* albedo, const double* emissive, const double* lightScale, uint32_t materialCount,
                uint32_t lightCount, const double* target, double* lossOut, double* eOut, double* gradOut,
                int32_t threads) {
    Scene sc = to_scene(s);
    Lights L;
    L.data = l->data; L.dataLen = l->dataLen; L.lightCount = l->lightCount; L.clustered = l->clustered;
    AdjProblem A;
    A.sc = &sc;
    A.L = &L;
    A.g = to_grid(g);
    std::memcpy(&A.P, params, sizeof(Params));
    A.tri = tri; A.inst = inst; A.blocked = blocked;
    A.solves = solves;
    A.roundAtlas = roundAtlas != 0;
    A.materialCount = materialCount;
    A.lightCount = lightCount;
    A.albedo = albedo; A.emissive = emissive; A.lightScale = lightScale;
    A.threads = std::max(1, (int)threads);
    AdjTape T;
    double loss = adj_forward(A, T, target);
    if (lossOut) *lossOut = loss;
    if (eOut) std::memcpy(eOut, T.E.data(), T.E.size() * sizeof(double));
    if (gradOut && target) adj_backward(A, T, target, gradOut);
    return 0;
}

}  // extern "C"
