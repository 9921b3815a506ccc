// sb_trace.cu — probe ray trace + hit shading (traceKernel, gi_probes.js:1977-2214)
// over the two-level BVH (spectral_traverse.js:354-569), for sm_100a.
//
// One thread per (probe slot, ray). Warps pull 32-ray batches from a global
// work counter (persistent, work-stealing), the TLAS is staged in shared
// memory, BLAS nodes / pre-gathered triangles are read as 16-byte vectors.
#include "sb_math.cuh"
#include "sb_kernels.cuh"

namespace sb {

struct TraceCtx {
    DevScene S;
    DevCascade C;
    DevParams P;
    uint32_t* err;
    unsigned long long* counters;  // [rays, shadowRays, tlasNodes, instances, blasNodes, triTests] or null
    uint32_t* work;                // work-stealing cursor (reset to 0 before launch)
    uint32_t totalRays;
    uint32_t smemTlas;             // TLAS nodes staged in shared memory
};

struct Visits { uint32_t tlas, inst, blas, tri; };

__device__ __forceinline__ bool slab(float3 bmin, float3 bmax, float3 ro, float3 invD, float tlim) {
    float t0x = (bmin.x - ro.x) * invD.x, t1x = (bmax.x - ro.x) * invD.x;
    float t0y = (bmin.y - ro.y) * invD.y, t1y = (bmax.y - ro.y) * invD.y;
    float t0z = (bmin.z - ro.z) * invD.z, t1z = (bmax.z - ro.z) * invD.z;
    float tNear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    float tFar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    return tFar >= fmaxf(tNear, 0.0f) && tNear < tlim;
}

__device__ __forceinline__ void load_node(const uint4* nodes, uint32_t c, float3& bmin, float3& bmax, uint32_t& miss,
                                          uint32_t& payload) {
    uint4 a = __ldg(nodes + 2 * c), b = __ldg(nodes + 2 * c + 1);
    bmin = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
    bmax = mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y));
    miss = b.z;
    payload = b.w;
}

// Möller–Trumbore on a pre-gathered triangle, spectral_traverse.js:393-409.
__device__ __forceinline__ bool mt_hit(const float4* tris, uint32_t tri, float3 ro, float3 rd, float tmax, float& t,
                                       float& det, float& u, float& v, uint32_t& bits) {
    float4 a = __ldg(tris + 3 * tri), b = __ldg(tris + 3 * tri + 1), c = __ldg(tris + 3 * tri + 2);
    float3 p0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
    float3 pv = cross3(rd, e2);
    det = dot3(e1, pv);
    if (!(fabsf(det) > 1e-12f)) return false;
    float invDet = 1.0f / det;
    float3 tv = ro - p0;
    u = dot3(tv, pv) * invDet;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    float3 qv = cross3(tv, e1);
    v = dot3(rd, qv) * invDet;
    if (!(v >= 0.0f && u + v <= 1.0f)) return false;
    t = dot3(e2, qv) * invDet;
    bits = __float_as_uint(a.w);
    return t > RAY_EPS && t < tmax;
}

__device__ __forceinline__ bool side_ok(uint32_t bits, float det) {
    uint32_t side = bits & TB_SIDE_MASK;
    return side == 2u || (side == 0u && det > 0.0f) || (side == 1u && det < 0.0f);
}

struct InstRay { float3 ro, rd, invD; uint32_t root, end; float dSign; };

__device__ __forceinline__ InstRay inst_ray(const float4* inst, uint32_t i, float3 wro, float3 wrd) {
    float4 r0 = __ldg(inst + 4 * i), r1 = __ldg(inst + 4 * i + 1), r2 = __ldg(inst + 4 * i + 2), m = __ldg(inst + 4 * i + 3);
    InstRay r;
    r.ro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
    r.rd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
    r.invD = mk(1.0f / r.rd.x, 1.0f / r.rd.y, 1.0f / r.rd.z);
    r.root = __float_as_uint(m.x);
    r.end = __float_as_uint(m.y);
    r.dSign = m.z;
    return r;
}

// blasClosest, spectral_traverse.js:354-435 (threaded, left-first).
__device__ __forceinline__ void blas_closest(const DevScene& S, uint32_t inst, float3 wro, float3 wrd, float& bestT,
                                             int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                             uint32_t* err) {
    InstRay r = inst_ray(S.inst, inst, wro, wrd);
    uint32_t cursor = r.root;
    uint32_t it = 0;
    for (; it < S.nodeCount; ++it) {
        if (cursor >= r.end) break;
        float3 bmin, bmax;
        uint32_t miss, payload;
        load_node(S.nodes, cursor, bmin, bmax, miss, payload);
        ++vis.blas;
        if (slab(bmin, bmax, r.ro, r.invD, bestT)) {
            if (payload == INTERIOR) {
                cursor = cursor + 1;
            } else {
                uint32_t off = payload & 0x00FFFFFFu, cnt = payload >> 24;
                for (uint32_t i = 0; i < cnt; ++i) {
                    uint32_t tri = off + i;
                    float t, det, u, v;
                    uint32_t bits;
                    ++vis.tri;
                    if (!mt_hit(S.tris, tri, r.ro, r.rd, bestT, t, det, u, v, bits)) continue;
                    if (side_ok(bits, det * r.dSign) && (bits & TB_CLOSEST_OK)) {
                        bestT = t;
                        bestTri = (int)tri;
                        bestInst = (int)inst;
                        bu = u;
                        bv = v;
                    }
                }
                cursor = miss;
            }
        } else {
            cursor = miss;
        }
    }
    if (it == S.nodeCount && cursor < r.end) latch(err, ERR_WATCHDOG);
}

__device__ __forceinline__ void load_tlas(const uint4* tl, uint32_t c, float3& bmin, float3& bmax, uint32_t& miss,
                                          uint32_t& payload) {
    uint4 a = tl[2 * c], b = tl[2 * c + 1];
    bmin = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
    bmax = mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y));
    miss = b.z;
    payload = b.w;
}

// traverseClosest, spectral_traverse.js:441-474
__device__ void trace_closest(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float& bestT, int& bestTri,
                              int& bestInst, float& bu, float& bv, Visits& vis, uint32_t* err) {
    bestT = T_MAX;
    bestTri = -1;
    bestInst = -1;
    bu = bv = 0.0f;
    float3 invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    uint32_t cursor = 0;
    for (uint32_t it = 0; it < S.tlasNodeCount; ++it) {
        if (cursor >= S.tlasNodeCount) break;
        float3 bmin, bmax;
        uint32_t miss, payload;
        load_tlas(tl, cursor, bmin, bmax, miss, payload);
        ++vis.tlas;
        if (slab(bmin, bmax, ro, invD, bestT)) {
            uint32_t cnt = payload >> 24;
            if (cnt == 0) {
                cursor = cursor + 1;
            } else {
                uint32_t off = payload & 0x00FFFFFFu;
                for (uint32_t i = 0; i < cnt; ++i) {
                    uint32_t inst = off + i;
                    ++vis.inst;
                    if (__ldg(&S.inst[4 * inst + 3].w) > 0.5f)
                        blas_closest(S, inst, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err);
                }
                cursor = miss;
            }
        } else {
            cursor = miss;
        }
    }
}

// The chosen hit's ray parameter re-evaluated in double-float: the same
// Möller–Trumbore expression (spectral_traverse.js:396-408) on the local ray
// (instLocalRay, 149-153), with the edges taken exactly from the pooled
// vertices. FP32 alone loses ~1e-5 relative on near hits (the local origin is
// rounded at scene scale); this keeps t within ~1e-7 of the exact value.
__device__ float refine_t(const DevScene& S, uint32_t tri, uint32_t inst, float3 wro, float3 wrd) {
    float4 r[3] = {__ldg(S.inst + 4 * inst), __ldg(S.inst + 4 * inst + 1), __ldg(S.inst + 4 * inst + 2)};
    dfl lo[3], ld[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = df_add(df_add(df_add(two_prod(r[k].x, wro.x), two_prod(r[k].y, wro.y)), two_prod(r[k].z, wro.z)),
                       df(r[k].w));
        ld[k] = df_add(df_add(two_prod(r[k].x, wrd.x), two_prod(r[k].y, wrd.y)), two_prod(r[k].z, wrd.z));
    }
    const float* p[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) p[k] = S.vertexData + (size_t)__ldg(S.triIndex + 3 * tri + k) * 8u;
    df3 p0 = {df(__ldg(p[0])), df(__ldg(p[0] + 1)), df(__ldg(p[0] + 2))};
    df3 p1 = {df(__ldg(p[1])), df(__ldg(p[1] + 1)), df(__ldg(p[1] + 2))};
    df3 p2 = {df(__ldg(p[2])), df(__ldg(p[2] + 1)), df(__ldg(p[2] + 2))};
    df3 e1 = df3_sub(p1, p0), e2 = df3_sub(p2, p0);
    df3 o = {lo[0], lo[1], lo[2]}, d = {ld[0], ld[1], ld[2]};
    df3 pv = df3_cross(d, e2);
    dfl det = df3_dot(e1, pv);
    df3 tv = df3_sub(o, p0);
    df3 qv = df3_cross(tv, e1);
    return df_div(df3_dot(e2, qv), det);
}

// blasAny, spectral_traverse.js:477-536
__device__ __forceinline__ bool blas_any(const DevScene& S, uint32_t inst, float3 wro, float3 wrd, float maxDist,
                                         Visits& vis, uint32_t* err) {
    InstRay r = inst_ray(S.inst, inst, wro, wrd);
    uint32_t cursor = r.root;
    uint32_t it = 0;
    for (; it < S.nodeCount; ++it) {
        if (cursor >= r.end) break;
        float3 bmin, bmax;
        uint32_t miss, payload;
        load_node(S.nodes, cursor, bmin, bmax, miss, payload);
        ++vis.blas;
        if (slab(bmin, bmax, r.ro, r.invD, maxDist)) {
            if (payload == INTERIOR) {
                cursor = cursor + 1;
            } else {
                uint32_t off = payload & 0x00FFFFFFu, cnt = payload >> 24;
                for (uint32_t i = 0; i < cnt; ++i) {
                    float t, det, u, v;
                    uint32_t bits;
                    ++vis.tri;
                    if (!mt_hit(S.tris, off + i, r.ro, r.rd, maxDist, t, det, u, v, bits)) continue;
                    if ((bits & TB_SHADOW_OK) && side_ok(bits, det * r.dSign)) return true;
                }
                cursor = miss;
            }
        } else {
            cursor = miss;
        }
    }
    if (it == S.nodeCount && cursor < r.end) latch(err, ERR_WATCHDOG);
    return false;
}

// traverseAny, spectral_traverse.js:539-569
__device__ bool trace_any(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float maxDist, Visits& vis,
                          uint32_t* err) {
    float3 invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    uint32_t cursor = 0;
    for (uint32_t it = 0; it < S.tlasNodeCount; ++it) {
        if (cursor >= S.tlasNodeCount) break;
        float3 bmin, bmax;
        uint32_t miss, payload;
        load_tlas(tl, cursor, bmin, bmax, miss, payload);
        ++vis.tlas;
        if (slab(bmin, bmax, ro, invD, maxDist)) {
            uint32_t cnt = payload >> 24;
            if (cnt == 0) {
                cursor = cursor + 1;
            } else {
                uint32_t off = payload & 0x00FFFFFFu;
                for (uint32_t i = 0; i < cnt; ++i) {
                    uint32_t inst = off + i;
                    ++vis.inst;
                    if (__ldg(&S.inst[4 * inst + 3].w) > 0.5f && blas_any(S, inst, ro, rd, maxDist, vis, err))
                        return true;
                }
                cursor = miss;
            }
        } else {
            cursor = miss;
        }
    }
    return false;
}

// sampleAtlas, gi_probes.js:1941-1974: 8-tap trilinear over the cage probes,
// each tap a bilinear fetch of the previous RGBA16F atlas (exact weights).
__device__ float3 sample_atlas(const DevCascade& C, float3 P, float3 N) {
    float3 cell = mk(C.gridSize[0] / fmaxf(1.0f, float(C.res[0]) - 1.0f),
                     C.gridSize[1] / fmaxf(1.0f, float(C.res[1]) - 1.0f),
                     C.gridSize[2] / fmaxf(1.0f, float(C.res[2]) - 1.0f));
    float gf[3] = {(P.x - C.gridMin[0]) / fmaxf(cell.x, 1e-6f), (P.y - C.gridMin[1]) / fmaxf(cell.y, 1e-6f),
                   (P.z - C.gridMin[2]) / fmaxf(cell.z, 1e-6f)};
    float base[3], frac[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        base[a] = clampf(floorf(gf[a]), 0.0f, fmaxf(float(C.res[a]) - 2.0f, 0.0f));
        frac[a] = clampf(gf[a] - base[a], 0.0f, 1.0f);
    }
    float2 ouv = oct_encode(normalize3(N));
    float3 acc = mk(0.f, 0.f, 0.f);
    float wsum = 0.0f;
    const float W = float(C.atlasW), H = float(C.atlasH);
    const int Wi = (int)C.atlasW, Hi = (int)C.atlasH;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        float px = base[0] + float(dx), py = base[1] + float(dy), pz = base[2] + float(dz);
        float wx = dx ? frac[0] : 1.0f - frac[0];
        float wy = dy ? frac[1] : 1.0f - frac[1];
        float wz = dz ? frac[2] : 1.0f - frac[2];
        float w = wx * wy * wz + 1e-4f;
        float row = pz * float(C.res[1]) + py;
        float ox = px * 8.0f + 1.0f + ouv.x * 6.0f;
        float oy = row * 8.0f + 1.0f + ouv.y * 6.0f;
        float x = (ox / W) * W - 0.5f, y = (oy / H) * H - 0.5f;
        float fx0 = floorf(x), fy0 = floorf(y);
        float fx = x - fx0, fy = y - fy0;
        int x0 = (int)fx0, y0 = (int)fy0;
        int xa = min(max(x0, 0), Wi - 1), xb = min(max(x0 + 1, 0), Wi - 1);
        int ya = min(max(y0, 0), Hi - 1), yb = min(max(y0 + 1, 0), Hi - 1);
        float4 t00 = half4_to_float4(__ldg(C.atlasPrev + (size_t)ya * Wi + xa));
        float4 t10 = half4_to_float4(__ldg(C.atlasPrev + (size_t)ya * Wi + xb));
        float4 t01 = half4_to_float4(__ldg(C.atlasPrev + (size_t)yb * Wi + xa));
        float4 t11 = half4_to_float4(__ldg(C.atlasPrev + (size_t)yb * Wi + xb));
        float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy), w01 = (1.0f - fx) * fy, w11 = fx * fy;
        float3 s = mk(t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11,
                      t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11,
                      t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11);
        acc = acc + s * w;
        wsum += w;
    }
    return acc * (1.0f / fmaxf(wsum, 1e-4f));
}

// shadeLight: NEE for one light, gi_probes.js:2065-2107 / 2130-2175.
__device__ __forceinline__ void shade_light(const TraceCtx& T, const uint4* tl, uint32_t li, float3 hitPos, float3 ng,
                                            float3 kd, float traceBias, float3& radiance, uint2& blockedBits,
                                            uint32_t& shadowRays, Visits& vis) {
    const float* L = T.S.lights + li * 17u;
    float ltype = __ldg(L);
    if (!(ltype < 2.5f)) return;
    float3 lpos = mk(__ldg(L + 1), __ldg(L + 2), __ldg(L + 3));
    float3 ldir = mk(__ldg(L + 4), __ldg(L + 5), __ldg(L + 6));
    float eclass = __ldg(L + 16);
    bool isIr = fabsf(eclass - 4.0f) < 0.25f;
    float irs = isIr ? T.P.nirGate * T.P.nirGain : 1.0f;
    float3 lcol = mk(__ldg(L + 7), __ldg(L + 8), __ldg(L + 9)) * irs;
    float lrange = __ldg(L + 10), ldecay = __ldg(L + 11), lcosAngle = __ldg(L + 12), lcosPen = __ldg(L + 13);
    bool isDir = ltype < 0.5f;
    bool isSpot = fabsf(ltype - 2.0f) < 0.5f;
    float3 toLight = isDir ? ldir * -1.0f : lpos - hitPos;
    float dist = isDir ? 1e4f : fmaxf(sqrtf(dot3(toLight, toLight)), 1e-4f);
    float3 wi = normalize3(toLight);
    float ndl = fmaxf(dot3(ng, wi), 0.0f);
    float lpeak = fmaxf(fmaxf(lcol.x, lcol.y), lcol.z);
    if (!(ndl * lpeak > 0.0f && (isDir || lrange <= 0.0f || dist < lrange))) return;
    ++shadowRays;
    bool blocked = trace_any(T.S, tl, hitPos, wi, dist - traceBias, vis, T.err);
    if (blocked) {
        if (li < 32) blockedBits.x |= 1u << li;
        else blockedBits.y |= 1u << (li - 32);
        return;
    }
    float falloff = 1.0f / fmaxf(powf(dist, ldecay), 0.01f);
    float rr = dist / fmaxf(lrange, 1e-4f);
    float rr2 = rr * rr;
    float win = clampf(1.0f - rr2 * rr2, 0.0f, 1.0f);
    float ranged = falloff * (win * win);
    float posAtten = lrange > 0.0f ? ranged : falloff;
    float distAtten = isDir ? 1.0f : posAtten;
    float angleCos = dot3(wi, ldir) * -1.0f;
    float spotAtten = clampf((angleCos - lcosAngle) / fmaxf(lcosPen - lcosAngle, 1e-4f), 0.0f, 1.0f);
    float atten = distAtten * (isSpot ? spotAtten : 1.0f);
    float3 diffuse = kd * (1.0f / PI_F);
    radiance = radiance + mul3(diffuse * ndl, lcol) * atten * T.P.debugDirectScale;
}

__device__ __forceinline__ float3 sky_sh(const DevParams& P, float3 rd) {
    float x = rd.x, y = rd.y, z = rd.z;
    float b[9] = {0.282095f, y * 0.488603f, z * 0.488603f, x * 0.488603f, x * y * 1.092548f, y * z * 1.092548f,
                  (z * z * 3.0f - 1.0f) * 0.315392f, x * z * 1.092548f, (x * x - y * y) * 0.546274f};
    float3 s = mk(0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 9; ++i) s = s + mk(P.skySH[3 * i], P.skySH[3 * i + 1], P.skySH[3 * i + 2]) * b[i];
    return mk(fmaxf(s.x, 0.f), fmaxf(s.y, 0.f), fmaxf(s.z, 0.f)) * P.skyIntensity;
}

__device__ void trace_one(const TraceCtx& T, const uint4* tl, uint32_t gid, Visits& vis, uint32_t& shadowRays) {
    const DevCascade& C = T.C;
    const uint32_t N = C.rays;
    uint32_t slot = gid / N, k = gid - slot * N;
    uint32_t probeIndex = (C.probeOffset + slot) % C.probeTotal;
    float3 ro = probe_world_pos(C, probeIndex);
    float3 rd = ray_dir(k, N, T.P.frameJitter);
    float bestT, bu, bv;
    int bestTri, bestInst;
    trace_closest(T.S, tl, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, T.err);
    float3 outRgb;
    float hitT = -1.0f;
    uint2 blockedBits = make_uint2(0u, 0u);
    if (bestTri >= 0) {
        uint32_t tri = (uint32_t)bestTri, inst = (uint32_t)bestInst;
        bestT = refine_t(T.S, tri, inst, ro, rd);
        hitT = bestT;
        uint32_t m = __ldg(T.S.triMaterial + tri);
        float4 b = __ldg(T.S.tris + 3 * tri + 1), c = __ldg(T.S.tris + 3 * tri + 2);
        float3 nl = normalize3(cross3(xyz(b), xyz(c)));
        float4 r0 = __ldg(T.S.inst + 4 * inst), r1 = __ldg(T.S.inst + 4 * inst + 1), r2 = __ldg(T.S.inst + 4 * inst + 2);
        float3 ngRaw = normalize3(xyz(r0) * nl.x + xyz(r1) * nl.y + xyz(r2) * nl.z);
        bool faceFwd = dot3(ngRaw, rd) < 0.0f;
        float3 ng = ngRaw * (faceFwd ? 1.0f : -1.0f);
        float3 hitPoint = ro + rd * bestT;
        float traceBias = fmaxf(C.cellMin * 0.005f * T.P.debugTraceBiasScale, RAY_EPS * T.P.debugRayEpsScale);
        float3 hitPos = hitPoint + ng * traceBias;
        const float* M = T.S.materials + (size_t)m * 28u;
        float3 baseColor = mk(__ldg(M), __ldg(M + 1), __ldg(M + 2));
        float3 emissive = mk(__ldg(M + 7), __ldg(M + 8), __ldg(M + 9));
        float3 radiance = emissive * T.P.debugEmissiveScale;
        float metal = __ldg(M + 4), transm = __ldg(M + 5);
        float3 kdr = baseColor * T.P.debugAlbedoScale * (1.0f - metal) * (1.0f - transm);
        float3 kd = mk(clampf(kdr.x, 0.f, 0.95f), clampf(kdr.y, 0.f, 0.95f), clampf(kdr.z, 0.f, 0.95f));
        if (T.S.clustered) {
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
            const float* list = T.S.lights + LIGHT_DATA + cellIndex * 17u;
            uint32_t listCount = (uint32_t)__ldg(list);
            if (outside || listCount > 16u) {
                for (uint32_t li = 0; li < T.S.lightCount; ++li)
                    shade_light(T, tl, li, hitPos, ng, kd, traceBias, radiance, blockedBits, shadowRays, vis);
            } else {
                for (uint32_t i = 0; i < listCount; ++i)
                    shade_light(T, tl, (uint32_t)__ldg(list + 1 + i), hitPos, ng, kd, traceBias, radiance, blockedBits,
                                shadowRays, vis);
            }
        } else {
            for (uint32_t li = 0; li < T.S.lightCount; ++li)
                shade_light(T, tl, li, hitPos, ng, kd, traceBias, radiance, blockedBits, shadowRays, vis);
        }
        float3 bounce = mul3(sample_atlas(C, hitPos, ng), kd) * (1.0f / PI_F);
        float bl = luma3(bounce);
        float roll = T.P.radianceClamp / fmaxf(fmaxf(T.P.radianceClamp, bl), 1e-6f);
        radiance = radiance + bounce * roll * T.P.debugBounceScale;
        outRgb = radiance;
        if (C.hits) {
            uint32_t uq = (uint32_t)__float2uint_rn(clampf(bu, 0.f, 1.f) * 65535.0f);
            uint32_t vq = (uint32_t)__float2uint_rn(clampf(bv, 0.f, 1.f) * 65535.0f);
            // bit 31 of the instance word records the facing decision (normal flipped or not)
            C.hits[gid] = make_uint4(tri, inst | (faceFwd ? 0x80000000u : 0u), __float_as_uint(bestT), uq | (vq << 16));
        }
    } else {
        outRgb = sky_sh(T.P, rd);
        if (C.hits) C.hits[gid] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, __float_as_uint(-1.0f), 0u);
    }
    if (C.vis) C.vis[gid] = blockedBits;
    C.rayData[gid] = make_float4(outRgb.x, outRgb.y, outRgb.z, hitT);
}

__global__ void __launch_bounds__(256) k_trace_shade(TraceCtx T) {
    extern __shared__ uint4 sTlas[];
    const DevScene& S = T.S;
    const uint4* tl = S.tlas;
    if (T.smemTlas >= S.tlasNodeCount && S.tlasNodeCount > 0) {
        for (uint32_t i = threadIdx.x; i < 2 * S.tlasNodeCount; i += blockDim.x) sTlas[i] = __ldg(S.tlas + i);
        __syncthreads();
        tl = sTlas;
    }
    if (!*S.valid) return;
    Visits vis = {0, 0, 0, 0};
    uint32_t shadowRays = 0, rays = 0;
    const uint32_t lane = threadIdx.x & 31u;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(T.work, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= T.totalRays) break;
        uint32_t gid = base + lane;
        if (gid < T.totalRays) {
            trace_one(T, tl, gid, vis, shadowRays);
            ++rays;
        }
    }
    if (T.counters) {
        atomicAdd(&T.counters[0], (unsigned long long)rays);
        atomicAdd(&T.counters[1], (unsigned long long)shadowRays);
        atomicAdd(&T.counters[2], (unsigned long long)vis.tlas);
        atomicAdd(&T.counters[3], (unsigned long long)vis.inst);
        atomicAdd(&T.counters[4], (unsigned long long)vis.blas);
        atomicAdd(&T.counters[5], (unsigned long long)vis.tri);
    }
}

cudaError_t launch_trace(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t* err,
                         unsigned long long* counters, uint32_t* work, const TraceTuning& tune, cudaStream_t st) {
    TraceCtx T;
    T.S = S;
    T.C = C;
    T.P = P;
    T.err = err;
    T.counters = counters;
    T.work = work;
    T.totalRays = C.updatedCount * C.rays;
    if (T.totalRays == 0) return cudaSuccess;
    uint32_t smemNodes = S.tlasNodeCount <= tune.smemTlasNodes ? S.tlasNodeCount : 0u;
    T.smemTlas = smemNodes ? smemNodes : 0u;
    size_t smem = (size_t)smemNodes * 32u;
    if (smem > 48u * 1024u) {
        cudaFuncSetAttribute(k_trace_shade, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    cudaMemsetAsync(work, 0, sizeof(uint32_t), st);
    int block = (int)tune.block;
    int blocksPerSm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSm, k_trace_shade, block, smem);
    if (blocksPerSm < 1) blocksPerSm = 1;
    int grid = tune.numSms * blocksPerSm;
    uint32_t needed = (T.totalRays + block - 1) / block;
    if ((uint32_t)grid > needed) grid = (int)needed;
    k_trace_shade<<<grid, block, smem, st>>>(T); note_launch();
    return cudaGetLastError();
}

// Arbitrary rays through traverseClosest / traverseAny (global TLAS reads).
__global__ void k_raycast(DevScene S, const float* ro, const float* rd, uint32_t n, float* tOut, int32_t* triOut,
                          int32_t* instOut, uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !*S.valid) return;
    Visits vis = {0, 0, 0, 0};
    float t, bu, bv;
    int tri, inst;
    float3 o = mk(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]), d = mk(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]);
    trace_closest(S, S.tlas, o, d, t, tri, inst, bu, bv, vis, err);
    if (tri >= 0) t = refine_t(S, (uint32_t)tri, (uint32_t)inst, o, d);
    tOut[i] = t;
    triOut[i] = tri;
    instOut[i] = inst;
}

__global__ void k_occluded(DevScene S, const float* ro, const float* rd, const float* maxDist, uint32_t n, uint8_t* out,
                           uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !*S.valid) return;
    Visits vis = {0, 0, 0, 0};
    out[i] = trace_any(S, S.tlas, mk(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]), mk(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]),
                       maxDist[i], vis, err)
                 ? 1
                 : 0;
}

cudaError_t launch_raycast(const DevScene& S, const float* ro, const float* rd, uint32_t n, float* tOut,
                           int32_t* triOut, int32_t* instOut, uint32_t* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_raycast<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, n, tOut, triOut, instOut, err); note_launch();
    return cudaGetLastError();
}

cudaError_t launch_occluded(const DevScene& S, const float* ro, const float* rd, const float* maxDist, uint32_t n,
                            uint8_t* out, uint32_t* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_occluded<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, maxDist, n, out, err); note_launch();
    return cudaGetLastError();
}

}  // namespace sb
