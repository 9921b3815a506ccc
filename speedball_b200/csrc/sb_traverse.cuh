// sb_traverse.cuh — two-level stackless traversal over the threaded BVH
// (spectral_traverse.js:354-569): closest hit and any hit, the double-float
// refinement of the final hit parameter, and the one-bounce atlas read
// (sampleAtlas, gi_probes.js:1941-1974). BLAS nodes and pre-gathered
// triangles are read as 16-byte vectors; the TLAS may be staged in shared memory.
#pragma once
#include "sb_math.cuh"
#include "sb_kernels.cuh"

namespace sb {

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
static __device__ __forceinline__ void trace_closest(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float& bestT, int& bestTri,
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
static __device__ float refine_t(const DevScene& S, uint32_t tri, uint32_t inst, float3 wro, float3 wrd) {
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
static __device__ __forceinline__ bool trace_any(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float maxDist, Visits& vis,
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
static __device__ float3 sample_atlas(const DevCascade& C, float3 P, float3 N) {
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


}  // namespace sb
