// sb_traverse.cuh — the closest-hit and any-hit queries (traverseClosest /
// traverseAny, spectral_traverse.js:354-569), the double-float refinement of
// the final hit parameter, and the one-bounce atlas read (sampleAtlas,
// gi_probes.js:1941-1974). Three walks answer the same query:
//   flat_walk   the scene BVH (default): one world-space tree over
//               (triangle, instance) items, local-space hit tests;
//   pair_walk   the reference's TLAS + BLASes as child-pair nodes, near first;
//   walk / nested_walk  the reference's threaded nodes in its own order.
// Every walk decides each (triangle, instance) pair with the reference's test.
//
// The reference nests a BLAS walk inside the TLAS walk. Here both levels run in
// one loop over the same 32-byte node encoding (bounds, miss link, payload), so
// lanes of a warp at different levels still execute the same node test, and
// leaf triangles are postponed until every lane of the warp holds a leaf (or is
// finished) so the triangle tests run together. The visiting order — left
// child first, TLAS leaf instances in slot order, first-visited wins ties — is
// the reference's, so hits, ties and visit counts are unchanged.
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

// Möller–Trumbore on a pre-gathered triangle, spectral_traverse.js:393-409.
// The triangle is stored as its three vertices; the edges are formed here with
// the same FP32 subtractions the reference's test makes.
__device__ __forceinline__ bool mt_hit(const float4* tris, uint32_t tri, float3 ro, float3 rd, float tmax, float& t,
                                       float& det, float& u, float& v, uint32_t& bits) {
    float4 a = __ldg(tris + 3 * tri), b = __ldg(tris + 3 * tri + 1), c = __ldg(tris + 3 * tri + 2);
    float3 p0 = xyz(a), e1 = xyz(b) - p0, e2 = xyz(c) - p0;
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

// Watertight ray/triangle test (Woop, Benthin & Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013): the vertices are translated to the ray
// origin and sheared so the ray runs along +z of a permuted frame (kz = the
// dominant axis of the direction, kx/ky swapped when it is negative to keep the
// winding); the three 2D edge functions of the projected triangle decide the
// hit. An edge shared by two triangles gets the same function value (negated)
// in both, since it is formed from the same two sheared vertices with the same
// separately rounded operations, so no ray passes between them; a value that
// comes out exactly zero is formed again in double precision. det = U + V + W
// has the sign of the Möller–Trumbore determinant (both are -dot(d, n) times a
// positive factor), so the reference's side test applies unchanged; (u, v) are
// the weights of vertices 1 and 2, as Möller–Trumbore's.
__device__ __forceinline__ bool wt_hit(const float4* tris, uint32_t tri, float3 ro, float3 rd, float tmax, float& t,
                                       float& det, float& u, float& v, uint32_t& bits) {
    const float4 a = __ldg(tris + 3 * tri), b = __ldg(tris + 3 * tri + 1), c = __ldg(tris + 3 * tri + 2);
    const float ax = fabsf(rd.x), ay = fabsf(rd.y), az = fabsf(rd.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
    const float d[3] = {rd.x, rd.y, rd.z};
    if (d[kz] < 0.0f) { const int tmp = kx; kx = ky; ky = tmp; }
    const float Sz = __frcp_rn(d[kz]);
    const float Sx = __fmul_rn(d[kx], Sz), Sy = __fmul_rn(d[ky], Sz);
    const float o[3] = {ro.x, ro.y, ro.z};
    const float A[3] = {__fsub_rn(a.x, o[0]), __fsub_rn(a.y, o[1]), __fsub_rn(a.z, o[2])};
    const float B[3] = {__fsub_rn(b.x, o[0]), __fsub_rn(b.y, o[1]), __fsub_rn(b.z, o[2])};
    const float C[3] = {__fsub_rn(c.x, o[0]), __fsub_rn(c.y, o[1]), __fsub_rn(c.z, o[2])};
    const float Ax = __fsub_rn(A[kx], __fmul_rn(Sx, A[kz])), Ay = __fsub_rn(A[ky], __fmul_rn(Sy, A[kz]));
    const float Bx = __fsub_rn(B[kx], __fmul_rn(Sx, B[kz])), By = __fsub_rn(B[ky], __fmul_rn(Sy, B[kz]));
    const float Cx = __fsub_rn(C[kx], __fmul_rn(Sx, C[kz])), Cy = __fsub_rn(C[ky], __fmul_rn(Sy, C[kz]));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    det = U + V + W;
    if (det == 0.0f) return false;
    const float T = __fmul_rn(Sz, U * A[kz] + V * B[kz] + W * C[kz]);
    const float inv = 1.0f / det;
    t = T * inv;
    u = V * inv;
    v = W * inv;
    bits = __float_as_uint(a.w);
    return t > RAY_EPS && t < tmax;
}

// The triangle test of this build: the reference's Möller–Trumbore (the
// parity default) or, built with SB_WATERTIGHT=1, the watertight test. A build
// switch rather than a runtime one: both tests inlined side by side in the
// traversal loops spill the closest-hit kernel's registers.
#ifndef SB_WATERTIGHT
#define SB_WATERTIGHT 0
#endif
__device__ __forceinline__ bool tri_hit(const DevScene& S, uint32_t tri, float3 ro, float3 rd, float tmax, float& t,
                                        float& det, float& u, float& v, uint32_t& bits) {
#if SB_WATERTIGHT
    return wt_hit(S.tris, tri, ro, rd, tmax, t, det, u, v, bits);
#else
    return mt_hit(S.tris, tri, ro, rd, tmax, t, det, u, v, bits);
#endif
}

// Both levels, one loop. ANY = traverseAny semantics (stop at the first
// accepted shadow-blocking hit inside tmax); otherwise traverseClosest
// (tmax shrinks to the nearest accepted hit).
template <bool ANY>
__device__ __forceinline__ bool walk(const DevScene& S, const uint4* tl, float3 wro, float3 wrd, float& tmax,
                                     int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis, uint32_t* err) {
    const float3 winv = mk(1.0f / wrd.x, 1.0f / wrd.y, 1.0f / wrd.z);
    float3 ro = wro, rd = wrd, invD = winv;
    uint32_t level = 0, cursor = 0, end = S.tlasNodeCount;
    uint32_t instNext = 0, instEnd = 0, tlResume = 0, inst = 0;
    float dSign = 1.0f;
    uint32_t iter = 0;
    for (;;) {
        uint32_t leafOff = 0, leafCnt = 0, leafMiss = 0;
        bool done = false;
        // node phase: walk until this lane holds a BLAS leaf or is finished
        for (;;) {
            if (level == 1 && cursor >= end) {
                bool entered = false;
                while (instNext < instEnd) {
                    uint32_t i = instNext++;
                    ++vis.inst;
                    float4 m = __ldg(S.inst + 4 * i + 3);
                    if (m.w > 0.5f) {  // active (spectral_traverse.js:464)
                        float4 r0 = __ldg(S.inst + 4 * i), r1 = __ldg(S.inst + 4 * i + 1), r2 = __ldg(S.inst + 4 * i + 2);
                        ro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
                        rd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
                        invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
                        cursor = __float_as_uint(m.x);
                        end = __float_as_uint(m.y);
                        dSign = m.z;
                        inst = i;
                        entered = true;
                        break;
                    }
                }
                if (!entered) {  // leaf done: resume the TLAS at its miss link
                    level = 0;
                    cursor = tlResume;
                    end = S.tlasNodeCount;
                    ro = wro;
                    rd = wrd;
                    invD = winv;
                }
                continue;
            }
            if (cursor >= end) {
                done = true;
                break;
            }
            if (++iter > S.iterCapRef) {
                latch(err, ERR_WATCHDOG);
                done = true;
                break;
            }
            uint4 a, b;
            if (level == 0) {
                a = tl[2 * cursor];
                b = tl[2 * cursor + 1];
                ++vis.tlas;
            } else {
                a = __ldg(S.nodes + 2 * cursor);
                b = __ldg(S.nodes + 2 * cursor + 1);
                ++vis.blas;
            }
            float3 bmin = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
            float3 bmax = mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y));
            if (!slab(bmin, bmax, ro, invD, tmax)) {
                cursor = b.z;
                continue;
            }
            if (level == 0) {
                uint32_t cnt = b.w >> 24;
                if (cnt == 0u) {
                    cursor = cursor + 1;
                } else {  // TLAS leaf: its instances in slot order, then the miss link
                    instNext = b.w & 0x00FFFFFFu;
                    instEnd = instNext + cnt;
                    tlResume = b.z;
                    level = 1;
                    cursor = end = 0;
                }
                continue;
            }
            if (b.w == INTERIOR) {
                cursor = cursor + 1;
                continue;
            }
            leafOff = b.w & 0x00FFFFFFu;
            leafCnt = b.w >> 24;
            leafMiss = b.z;
            break;
        }
        if (done) break;
        // leaf phase (warp-aligned)
        for (uint32_t i = 0; i < leafCnt; ++i) {
            uint32_t tri = leafOff + i;
            float t, det, u, v;
            uint32_t bits;
            ++vis.tri;
            if (!tri_hit(S, tri, ro, rd, tmax, t, det, u, v, bits)) continue;
            if (ANY) {
                if ((bits & TB_SHADOW_OK) && side_ok(bits, det * dSign)) return true;
            } else if (side_ok(bits, det * dSign) && (bits & TB_CLOSEST_OK)) {
                tmax = t;
                bestTri = (int)tri;
                bestInst = (int)inst;
                bu = u;
                bv = v;
            }
        }
        cursor = leafMiss;
    }
    return ANY ? false : bestTri >= 0;
}

// One BLAS (spectral_traverse.js:354-435 / 477-536) for the nested schedule.
// POSTPONE = while-while: walk interior nodes until a leaf, then test it.
template <bool ANY, bool POSTPONE>
__device__ __forceinline__ bool blas_walk(const DevScene& S, uint32_t inst, float3 wro, float3 wrd, float& tmax,
                                          int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                          uint32_t* err) {
    float4 r0 = __ldg(S.inst + 4 * inst), r1 = __ldg(S.inst + 4 * inst + 1), r2 = __ldg(S.inst + 4 * inst + 2),
           m = __ldg(S.inst + 4 * inst + 3);
    const float3 ro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
    const float3 rd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
    const float3 invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    uint32_t cursor = __float_as_uint(m.x);
    const uint32_t end = __float_as_uint(m.y);
    const float dSign = m.z;
    uint32_t it = 0;
    while (cursor < end) {
        uint32_t leafOff = 0, leafCnt = 0, leafMiss = 0;
        bool leaf = false;
        while (cursor < end) {
            if (++it > min(S.nodeCount, S.iterCapRef)) {
                latch(err, ERR_WATCHDOG);
                return ANY ? false : bestTri >= 0;
            }
            uint4 a = __ldg(S.nodes + 2 * cursor), b = __ldg(S.nodes + 2 * cursor + 1);
            ++vis.blas;
            float3 bmin = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
            float3 bmax = mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y));
            if (!slab(bmin, bmax, ro, invD, tmax)) {
                cursor = b.z;
            } else if (b.w == INTERIOR) {
                cursor = cursor + 1;
            } else {
                leafOff = b.w & 0x00FFFFFFu;
                leafCnt = b.w >> 24;
                leafMiss = b.z;
                leaf = true;
                if (POSTPONE) break;
                for (uint32_t i = 0; i < leafCnt; ++i) {
                    uint32_t tri = leafOff + i;
                    float t, det, u, v;
                    uint32_t bits;
                    ++vis.tri;
                    if (!tri_hit(S, tri, ro, rd, tmax, t, det, u, v, bits)) continue;
                    if (ANY) {
                        if ((bits & TB_SHADOW_OK) && side_ok(bits, det * dSign)) return true;
                    } else if (side_ok(bits, det * dSign) && (bits & TB_CLOSEST_OK)) {
                        tmax = t; bestTri = (int)tri; bestInst = (int)inst; bu = u; bv = v;
                    }
                }
                cursor = leafMiss;
                leaf = false;
            }
        }
        if constexpr (POSTPONE) {
            if (!leaf) break;
            for (uint32_t i = 0; i < leafCnt; ++i) {
                uint32_t tri = leafOff + i;
                float t, det, u, v;
                uint32_t bits;
                ++vis.tri;
                if (!tri_hit(S, tri, ro, rd, tmax, t, det, u, v, bits)) continue;
                if (ANY) {
                    if ((bits & TB_SHADOW_OK) && side_ok(bits, det * dSign)) return true;
                } else if (side_ok(bits, det * dSign) && (bits & TB_CLOSEST_OK)) {
                    tmax = t; bestTri = (int)tri; bestInst = (int)inst; bu = u; bv = v;
                }
            }
            cursor = leafMiss;
        } else {
            break;
        }
    }
    return ANY ? false : bestTri >= 0;
}

// The reference's nested schedule: TLAS walk, BLAS walk per active leaf instance.
template <bool ANY, bool POSTPONE>
__device__ __forceinline__ bool nested_walk(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float& tmax,
                                            int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                            uint32_t* err) {
    const float3 invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    uint32_t cursor = 0;
    for (uint32_t it = 0; it < S.tlasNodeCount && cursor < S.tlasNodeCount; ++it) {
        uint4 a = tl[2 * cursor], b = tl[2 * cursor + 1];
        ++vis.tlas;
        float3 bmin = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
        float3 bmax = mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y));
        if (!slab(bmin, bmax, ro, invD, tmax)) {
            cursor = b.z;
            continue;
        }
        uint32_t cnt = b.w >> 24;
        if (cnt == 0u) {
            cursor = cursor + 1;
            continue;
        }
        uint32_t off = b.w & 0x00FFFFFFu;
        for (uint32_t i = 0; i < cnt; ++i) {
            uint32_t inst = off + i;
            ++vis.inst;
            if (__ldg(&S.inst[4 * inst + 3].w) > 0.5f &&
                blas_walk<ANY, POSTPONE>(S, inst, ro, rd, tmax, bestTri, bestInst, bu, bv, vis, err) && ANY)
                return true;
        }
        cursor = b.z;
    }
    return ANY ? false : bestTri >= 0;
}

// ------------------------------------------------------ child-pair walk
// The same two-level query over the child-pair nodes: each step loads one
// 64-byte node, tests both children's boxes (the reference's slab test on the
// reference bounds), descends into the nearer hit child and stacks the other
// with its entry distance. A closest-hit query skips a stacked child once the
// nearest hit lies at or before that distance, which is exactly the reference's
// box test `tNear < tmax` evaluated again. Instances of a TLAS leaf still run in
// slot order, each from its BLAS root box. The hit is the reference's nearest
// accepted hit; among hits at exactly equal t the first one found wins, which
// can differ from the reference's left-first order only on such ties.

__device__ __forceinline__ bool slab_near(float bminx, float bminy, float bminz, float bmaxx, float bmaxy,
                                          float bmaxz, float3 ro, float3 invD, float tlim, float& tNearOut) {
    float t0x = (bminx - ro.x) * invD.x, t1x = (bmaxx - ro.x) * invD.x;
    float t0y = (bminy - ro.y) * invD.y, t1y = (bmaxy - ro.y) * invD.y;
    float t0z = (bminz - ro.z) * invD.z, t1z = (bmaxz - ro.z) * invD.z;
    float tNear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    float tFar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    tNearOut = tNear;
    return tFar >= fmaxf(tNear, 0.0f) && tNear < tlim;
}

// True when the pair layout is current and the deepest TLAS + BLAS path fits
// the stack (one stacked entry per level at most).
__device__ __forceinline__ bool pairs_usable(const DevScene& S) {
    if (!S.depth || !S.pairs || !S.tlasPairs) return false;
    uint32_t db = __ldg(S.depth), dt = __ldg(S.depth + 1);
    return db != DEPTH_UNKNOWN && dt != DEPTH_UNKNOWN && db + dt + 2u <= (uint32_t)SB_STACK;
}

template <bool ANY>
__device__ __forceinline__ bool pair_walk(const DevScene& S, const uint4* tp, float3 wro, float3 wrd, float& tmax,
                                          int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                          uint32_t* err) {
    const float3 winv = mk(1.0f / wrd.x, 1.0f / wrd.y, 1.0f / wrd.z);
    float3 ro = wro, rd = wrd, invD = winv;
    uint2 stk[SB_STACK];
    int sp = 0, blasBase = -1;
    uint32_t instNext = 0, instEnd = 0, inst = 0;
    float dSign = 1.0f;
    uint32_t cur = PE_NONE;
    if (S.tlasNodeCount == 0) return false;
    {  // the TLAS root box, as the reference's first TLAS step
        uint4 a = __ldg(S.tlas), b = __ldg(S.tlas + 1);
        ++vis.tlas;
        if (!slab(mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z)),
                  mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y)), ro, invD, tmax))
            return false;
        uint32_t cnt = b.w >> 24, slot = b.w & 0x00FFFFFFu;
        cur = cnt == 0u ? 0u : (slot < PE_TLAS_MAX_SLOTS && cnt < 1024u ? (PE_TLEAF | (cnt << 12) | slot) : PE_NONE);
    }
    uint32_t iter = 0;
    for (;;) {
        uint32_t leaf = PE_NONE;
        bool done = false;
        // node phase: until this lane holds a BLAS leaf or has nothing left
        for (;;) {
            if (cur == PE_NONE) {
                if (blasBase >= 0 && sp == blasBase) {
                    // this BLAS is done: the next active instance of the TLAS leaf
                    while (instNext < instEnd) {
                        uint32_t i = instNext++;
                        ++vis.inst;
                        float4 m = __ldg(S.inst + 4 * i + 3);
                        if (!(m.w > 0.5f)) continue;  // inactive (spectral_traverse.js:464)
                        float4 r0 = __ldg(S.inst + 4 * i), r1 = __ldg(S.inst + 4 * i + 1),
                               r2 = __ldg(S.inst + 4 * i + 2);
                        ro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
                        rd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
                        invD = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
                        uint32_t root = __float_as_uint(m.x);
                        uint4 a = __ldg(S.nodes + 2 * root), b = __ldg(S.nodes + 2 * root + 1);
                        ++vis.blas;
                        if (!slab(mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z)),
                                  mk(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y)), ro, invD,
                                  tmax))
                            continue;
                        cur = b.w == INTERIOR ? (root < PE_BLAS_MAX_NODES ? (PE_BLAS | root) : PE_NONE)
                                              : ((b.w >> 24) ? b.w : PE_NONE);
                        if (cur == PE_NONE) continue;
                        dSign = m.z;
                        inst = i;
                        break;
                    }
                    if (cur != PE_NONE) continue;
                    blasBase = -1;  // leaf exhausted: back to the TLAS
                    ro = wro;
                    rd = wrd;
                    invD = winv;
                }
                if (sp == 0) {
                    done = true;
                    break;
                }
                --sp;
                uint2 e = stk[sp];
                if (!ANY && __uint_as_float(e.y) >= tmax) continue;  // behind the nearest hit now
                cur = e.x;
            }
            if (++iter > S.iterCapRef) {
                latch(err, ERR_WATCHDOG);
                done = true;
                break;
            }
            if (cur >> 24) {  // BLAS leaf
                leaf = cur;
                cur = PE_NONE;
                break;
            }
            if ((cur & (PE_BLAS | PE_TLEAF)) == PE_TLEAF) {  // TLAS leaf: its instances in slot order
                instNext = cur & 0xFFFu;
                instEnd = instNext + ((cur >> 12) & 0x3FFu);
                blasBase = sp;
                cur = PE_NONE;
                continue;
            }
            uint4 q0, q1, q2, q3;
            if (cur & PE_BLAS) {
                const uint4* p = S.pairs + 4u * (cur & (PE_BLAS - 1u));
                q0 = __ldg(p); q1 = __ldg(p + 1); q2 = __ldg(p + 2); q3 = __ldg(p + 3);
                vis.blas += 2;
            } else {
                const uint4* p = tp + 4u * cur;
                q0 = p[0]; q1 = p[1]; q2 = p[2]; q3 = p[3];
                vis.tlas += 2;
            }
            float tn0 = 0.f, tn1 = 0.f;
            bool h0 = q3.x != PE_NONE &&
                      slab_near(__uint_as_float(q0.x), __uint_as_float(q0.z), __uint_as_float(q2.x),
                                __uint_as_float(q0.y), __uint_as_float(q0.w), __uint_as_float(q2.y), ro, invD, tmax, tn0);
            bool h1 = q3.y != PE_NONE &&
                      slab_near(__uint_as_float(q1.x), __uint_as_float(q1.z), __uint_as_float(q2.z),
                                __uint_as_float(q1.y), __uint_as_float(q1.w), __uint_as_float(q2.w), ro, invD, tmax, tn1);
            if (h0 && h1) {
                if (sp >= SB_STACK) {  // unreachable when pairs_usable() held
                    latch(err, ERR_CAPACITY);
                    done = true;
                    break;
                }
                const bool swap = tn1 < tn0;
                stk[sp++] = make_uint2(swap ? q3.x : q3.y, __float_as_uint(swap ? tn0 : tn1));
                cur = swap ? q3.y : q3.x;
            } else {
                cur = h0 ? q3.x : (h1 ? q3.y : PE_NONE);
            }
        }
        if (done) break;
        // leaf phase (warp-aligned)
        const uint32_t off = leaf & 0x00FFFFFFu, cnt = leaf >> 24;
        for (uint32_t i = 0; i < cnt; ++i) {
            uint32_t tri = off + i;
            float t, det, u, v;
            uint32_t bits;
            ++vis.tri;
            if (!tri_hit(S, tri, ro, rd, tmax, t, det, u, v, bits)) continue;
            if (ANY) {
                if ((bits & TB_SHADOW_OK) && side_ok(bits, det * dSign)) return true;
            } else if (side_ok(bits, det * dSign) && (bits & TB_CLOSEST_OK)) {
                tmax = t;
                bestTri = (int)tri;
                bestInst = (int)inst;
                bu = u;
                bv = v;
            }
        }
    }
    return ANY ? false : bestTri >= 0;
}

// ------------------------------------------------------ scene-BVH walk
// One world-space tree over (triangle, slot) items (sb_flat.h), near child
// first with a stack; a stacked child is skipped once the nearest hit lies at
// or before its entry distance. An item is tested in its instance's local space
// on the local ray the reference forms (instLocalRay, spectral_traverse.js:
// 149-153), with the reference's Möller–Trumbore and side/alpha acceptance, so
// each (triangle, instance) pair is accepted or rejected exactly as the
// reference's walk would. Slots moved or deformed since the tree was built are
// skipped there and walked through their current BLAS (reference order).
// Hits at exactly equal t may resolve to a different (triangle, instance) than
// the reference's left-first order; every other hit is the reference's.
constexpr uint32_t FLAT_LEAF = 0x80000000u;
constexpr uint32_t FLAT_NONE = 0xFFFFFFFFu;

// Moved slots walked before (1) or after (0) the tree. Measured on the atrium
// (one deforming slot): any hit 0.13 vs 0.42 ms, closest hit 0.41 vs 0.44 ms.
// After the tree, the any-hit early exits leave the lanes of a warp
// unconverged through the moved-slot walk (2.5 vs 10.5 active lanes per
// instruction for the same thread work).
#ifndef SB_DYN_FIRST
#define SB_DYN_FIRST 1
#endif

// A slot that left the tree: its world bounds (the reference's TLAS leaf
// test), then its BLAS in the reference's order.
template <bool ANY>
__device__ __forceinline__ bool dyn_walk(const DevScene& S, float3 wro, float3 wrd, float3 winv, float& tmax,
                                         int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                         uint32_t* err) {
    for (uint32_t k = 0; k < S.dynCount; ++k) {
        const uint32_t inst = __ldg(S.dynList + k);
        if (S.slotBounds) {
            const float* b = S.slotBounds + 6u * inst;
            if (!slab(mk(__ldg(b), __ldg(b + 1), __ldg(b + 2)), mk(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5)), wro,
                      winv, tmax))
                continue;
        }
        ++vis.inst;
        if (__ldg(&S.inst[4 * inst + 3].w) > 0.5f &&
            blas_walk<ANY, false>(S, inst, wro, wrd, tmax, bestTri, bestInst, bu, bv, vis, err) && ANY)
            return true;
    }
    return false;
}

template <bool ANY>
__device__ __forceinline__ bool flat_walk(const DevScene& S, float3 wro, float3 wrd, float& tmax, int& bestTri,
                                          int& bestInst, float& bu, float& bv, Visits& vis, uint32_t* err) {
    const float3 winv = mk(1.0f / wrd.x, 1.0f / wrd.y, 1.0f / wrd.z);
    if (SB_DYN_FIRST && dyn_walk<ANY>(S, wro, wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    uint2 stk[SB_STACK];
    int sp = 0;
    uint32_t cur = S.flatRoot;
    uint32_t lslot = FLAT_NONE;  // slot of the cached local ray
    float3 lro = wro, lrd = wrd;
    float dSign = 1.0f;
    uint32_t iter = 0;
    for (;;) {
        uint32_t leaf = FLAT_NONE;
        bool done = false;
        // node phase: until this lane holds a leaf or has nothing left
        for (;;) {
            if (cur == FLAT_NONE) {
                if (sp == 0) {
                    done = true;
                    break;
                }
                --sp;
                uint2 e = stk[sp];
                if (!ANY && __uint_as_float(e.y) >= tmax) continue;  // behind the nearest hit now
                cur = e.x;
            }
            if (cur & FLAT_LEAF) {
                leaf = cur;
                cur = FLAT_NONE;
                break;
            }
            if (++iter > S.iterCap) {
                latch(err, ERR_WATCHDOG);
                done = true;
                break;
            }
            const uint4* p = S.flatNodes + 4u * cur;
            const uint4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
            vis.blas += 2;
            float tn0 = 0.f, tn1 = 0.f;
            const bool h0 = slab_near(__uint_as_float(q0.x), __uint_as_float(q0.z), __uint_as_float(q2.x),
                                      __uint_as_float(q0.y), __uint_as_float(q0.w), __uint_as_float(q2.y), wro, winv,
                                      tmax, tn0) && q3.x != FLAT_NONE;
            const bool h1 = slab_near(__uint_as_float(q1.x), __uint_as_float(q1.z), __uint_as_float(q2.z),
                                      __uint_as_float(q1.y), __uint_as_float(q1.w), __uint_as_float(q2.w), wro, winv,
                                      tmax, tn1) && q3.y != FLAT_NONE;
            if (h0 && h1) {
                if (sp >= SB_STACK) {  // unreachable: the tree's depth was checked on build
                    latch(err, ERR_CAPACITY);
                    done = true;
                    break;
                }
                const bool swap = tn1 < tn0;
                stk[sp++] = make_uint2(swap ? q3.x : q3.y, __float_as_uint(swap ? tn0 : tn1));
                cur = swap ? q3.y : q3.x;
            } else {
                cur = h0 ? q3.x : (h1 ? q3.y : FLAT_NONE);
            }
        }
        if (done) break;
        // leaf phase (warp-aligned): items in slot order share the local ray
        const uint32_t first = leaf & 0x00FFFFFFu, cnt = (leaf >> 24) & 0x7Fu;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint2 it = __ldg(S.flatItems + first + k);
            const uint32_t tri = it.x, slot = it.y;
            if (slot != lslot) {
                if (__ldg(S.slotSkip + slot)) continue;
                const float4 r0 = __ldg(S.inst + 4 * slot), r1 = __ldg(S.inst + 4 * slot + 1),
                             r2 = __ldg(S.inst + 4 * slot + 2);
                lro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
                lrd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
                dSign = __ldg(&S.inst[4 * slot + 3].z);
                lslot = slot;
                ++vis.inst;
            }
            float t, det, u, v;
            uint32_t bits;
            ++vis.tri;
            if (!tri_hit(S, tri, lro, lrd, tmax, t, det, u, v, bits)) continue;
            if (ANY) {
                if ((bits & TB_SHADOW_OK) && side_ok(bits, det * dSign)) return true;
            } else if (side_ok(bits, det * dSign) && (bits & TB_CLOSEST_OK)) {
                tmax = t;
                bestTri = (int)tri;
                bestInst = (int)slot;
                bu = u;
                bv = v;
            }
        }
    }
    // after the tree, the nearest hit so far culls the moved slots
    if (!SB_DYN_FIRST && dyn_walk<ANY>(S, wro, wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    return ANY ? false : bestTri >= 0;
}

// ------------------------------------------------------ wide scene-BVH walk
// The scene BVH as 8-wide nodes with 8-bit child boxes (sb_flat.h). One node
// visit tests all eight child boxes and forms one hit mask: interior children
// at bit 24 + (slot XOR ray octant), so taking the lowest bit first visits
// them roughly near to far; leaf items at their offsets in bits 0..23. A
// group (child base, remaining interior bits, interior mask) waits on the stack
// while the nearest child is visited; a node's items are tested before its
// children. Box tests are conservative (outward-rounded grid, widened item
// bounds); the items are tested exactly as in flat_walk.

// q (a byte of w, 0..255) as an exact float: 2^23 + q minus 2^23
__device__ __forceinline__ float q_at(uint32_t w, uint32_t byteSel) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | byteSel)) - 8388608.0f;
}

// Box-test instruction forms of sm_100 (each exact, so the hit decisions are
// the same in every form): three-input min / max (PTX ISA 8.8), two children's
// plane distances per packed f32x2 add + fma (PTX ISA 8.6), and child hits
// gathered as an 8-bit slot mask turned into traversal bits once per node.
#ifndef SB_WIDE_MINMAX3
#define SB_WIDE_MINMAX3 1
#endif
#ifndef SB_WIDE_F32X2
#define SB_WIDE_F32X2 1
#endif
#ifndef SB_WIDE_HITMASK
#define SB_WIDE_HITMASK 1
#endif

__device__ __forceinline__ float max3f(float a, float b, float c) {
#if SB_WIDE_MINMAX3
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
#else
    return fmaxf(fmaxf(a, b), c);
#endif
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
#if SB_WIDE_MINMAX3
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
#else
    return fminf(fminf(a, b), c);
#endif
}

__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

// Plane distances of bytes b and b + 1 of w: q * s + o for both, where
// s2 = (s, s) and o2 = (o, o); per lane the same IEEE operations as
// fmaf(q_at(w, b), s, o).
__device__ __forceinline__ void q_pair(uint32_t w, uint32_t b, unsigned long long s2, unsigned long long o2, float& t0,
                                       float& t1) {
    const uint32_t a0 = __byte_perm(w, 0x4B000000u, 0x7540u | b);
    const uint32_t a1 = __byte_perm(w, 0x4B000000u, 0x7540u | (b + 1u));
    const unsigned long long bias = 0xCB000000CB000000ull;  // (-2^23, -2^23)
    unsigned long long r;
    asm("{\n\t.reg .b64 a;\n\tmov.b64 a, {%1, %2};\n\tadd.rn.f32x2 a, a, %3;\n\tfma.rn.f32x2 %0, a, %4, %5;\n\t}"
        : "=l"(r)
        : "r"(a0), "r"(a1), "l"(bias), "l"(s2), "l"(o2));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(t0), "=f"(t1) : "l"(r));
}

// One node visit of the 8-wide walk: its eight child boxes against the ray
// (nearer than tmax) -> the group of hit interior children (gBase; gBits holds
// the hits at bit 24 + (slot XOR octant) and the interior mask at bit 16) and
// the hit leaves' items (tBase, tBits).
__device__ __forceinline__ void wide_visit(const DevScene& S, uint32_t node, float3 wro, float3 binv, uint32_t oct,
                                           float tmax, const uint4* sWide, uint32_t nWide, Visits& vis,
                                           uint32_t& gBase, uint32_t& gBits, uint32_t& tBase, uint32_t& tBits) {
    uint4 h0, h1, qa, qb, qc;
    if (node < nWide) {
        const uint4* p = sWide + 5u * node;
        h0 = p[0];
        h1 = p[1];
        qa = p[2];
        qb = p[3];
        qc = p[4];
    } else {
        const uint4* p = S.wideNodes + 5u * node;
        h0 = __ldg(p);
        h1 = __ldg(p + 1);
        qa = __ldg(p + 2);
        qb = __ldg(p + 3);
        qc = __ldg(p + 4);
    }
    vis.blas += 8;
    // per axis: t = q * (2^e * inv) + (p - o) * inv, near plane first
    const float sx = __uint_as_float((h0.w & 0xFFu) << 23) * binv.x;
    const float sy = __uint_as_float(((h0.w >> 8) & 0xFFu) << 23) * binv.y;
    const float sz = __uint_as_float(((h0.w >> 16) & 0xFFu) << 23) * binv.z;
    const float ox = (__uint_as_float(h0.x) - wro.x) * binv.x;
    const float oy = (__uint_as_float(h0.y) - wro.y) * binv.y;
    const float oz = (__uint_as_float(h0.z) - wro.z) * binv.z;
    // lo words: x (qa.x, qa.y) y (qa.z, qa.w) z (qb.x, qb.y); hi words: x (qb.z, qb.w) y (qc.x, qc.y) z (qc.z, qc.w)
    const bool nx = oct & 1u, ny = oct & 2u, nz = oct & 4u;
    const uint32_t nearX0 = nx ? qb.z : qa.x, nearX1 = nx ? qb.w : qa.y;
    const uint32_t farX0 = nx ? qa.x : qb.z, farX1 = nx ? qa.y : qb.w;
    const uint32_t nearY0 = ny ? qc.x : qa.z, nearY1 = ny ? qc.y : qa.w;
    const uint32_t farY0 = ny ? qa.z : qc.x, farY1 = ny ? qa.w : qc.y;
    const uint32_t nearZ0 = nz ? qc.z : qb.x, nearZ1 = nz ? qc.w : qb.y;
    const uint32_t farZ0 = nz ? qb.x : qc.z, farZ1 = nz ? qb.y : qc.w;
    uint32_t bits = 0;  // hit mask over slots (SB_WIDE_HITMASK), else traversal bits
    // child s's box against the ray from its six plane distances
    auto child = [&](uint32_t s, float tnx, float tny, float tnz, float tfx, float tfy, float tfz) {
        const float tNear = max3f(tnx, tny, tnz);
        const float tFar = min3f(tfx, tfy, tfz);
        const bool hit = tFar >= fmaxf(tNear, 0.0f) && tNear < tmax;
#if SB_WIDE_HITMASK
        bits |= (hit ? 1u : 0u) << s;
#else
        if (hit) {
            const uint32_t m = (s < 4 ? h1.z : h1.w) >> (8u * (s & 3u)) & 0xFFu;
            uint32_t sh = m & 31u;
            if (sh >= 24u) sh ^= oct;
            bits |= (m >> 5) << sh;
        }
#endif
    };
#if SB_WIDE_F32X2
    const unsigned long long sx2 = pack2(sx, sx), sy2 = pack2(sy, sy), sz2 = pack2(sz, sz);
    const unsigned long long ox2 = pack2(ox, ox), oy2 = pack2(oy, oy), oz2 = pack2(oz, oz);
#pragma unroll
    for (uint32_t s = 0; s < 8; s += 2) {  // two children per packed operation
        const uint32_t b = s & 3u;
        float nx0, nx1, ny0, ny1, nz0, nz1, fx0, fx1, fy0, fy1, fz0, fz1;
        q_pair(s < 4 ? nearX0 : nearX1, b, sx2, ox2, nx0, nx1);
        q_pair(s < 4 ? nearY0 : nearY1, b, sy2, oy2, ny0, ny1);
        q_pair(s < 4 ? nearZ0 : nearZ1, b, sz2, oz2, nz0, nz1);
        q_pair(s < 4 ? farX0 : farX1, b, sx2, ox2, fx0, fx1);
        q_pair(s < 4 ? farY0 : farY1, b, sy2, oy2, fy0, fy1);
        q_pair(s < 4 ? farZ0 : farZ1, b, sz2, oz2, fz0, fz1);
        child(s, nx0, ny0, nz0, fx0, fy0, fz0);
        child(s + 1u, nx1, ny1, nz1, fx1, fy1, fz1);
    }
#else
#pragma unroll
    for (uint32_t s = 0; s < 8; ++s) {
        const uint32_t b = s & 3u;
        child(s, fmaf(q_at(s < 4 ? nearX0 : nearX1, b), sx, ox), fmaf(q_at(s < 4 ? nearY0 : nearY1, b), sy, oy),
              fmaf(q_at(s < 4 ? nearZ0 : nearZ1, b), sz, oz), fmaf(q_at(s < 4 ? farX0 : farX1, b), sx, ox),
              fmaf(q_at(s < 4 ? farY0 : farY1, b), sy, oy), fmaf(q_at(s < 4 ? farZ0 : farZ1, b), sz, oz));
    }
#endif
#if SB_WIDE_HITMASK
    {
        // interior hits to bit (slot XOR octant): visiting the lowest first goes near to far
        const uint32_t imask = h0.w >> 24;
        uint32_t ih = bits & imask;
        if (oct & 1u) ih = ((ih & 0x55u) << 1) | ((ih >> 1) & 0x55u);
        if (oct & 2u) ih = ((ih & 0x33u) << 2) | ((ih >> 2) & 0x33u);
        if (oct & 4u) ih = ((ih & 0x0Fu) << 4) | (ih >> 4);
        // leaf hits: each one's item bits at its offset
        uint32_t lh = bits & ~imask & 0xFFu, items = 0;
        while (lh) {
            const uint32_t s = __ffs(lh) - 1u;
            lh &= lh - 1u;
            const uint32_t m = __byte_perm(h1.z, h1.w, s) & 0xFFu;
            items |= (m >> 5) << (m & 31u);
        }
        bits = ih << 24 | items;
    }
#endif
    gBase = h1.x;
    gBits = (bits & 0xFF000000u) | ((h0.w >> 24) << 16);
    tBase = h1.y;
    tBits = bits & 0x00FFFFFFu;
}

// The items of the hit leaves (tBits over the run at tBase) against the ray,
// in slot order so that consecutive items share the local ray. True on an any
// hit (ANY); closest hits shrink tmax.
template <bool ANY>
__device__ __forceinline__ bool wide_items(const DevScene& S, uint32_t tBase, uint32_t tBits, float3 wro, float3 wrd,
                                           uint32_t& lslot, float3& lro, float3& lrd, float& dSign, float& tmax,
                                           int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis) {
    while (tBits) {
        const uint32_t k = __ffs(tBits) - 1u;
        tBits &= tBits - 1u;
        const uint2 it = __ldg(S.wideItems + tBase + k);
        const uint32_t tri = it.x, slot = it.y;
        if (slot != lslot) {
            if (__ldg(S.slotSkip + slot)) continue;
            const float4 r0 = __ldg(S.inst + 4 * slot), r1 = __ldg(S.inst + 4 * slot + 1),
                         r2 = __ldg(S.inst + 4 * slot + 2);
            lro = mk(dot3(xyz(r0), wro) + r0.w, dot3(xyz(r1), wro) + r1.w, dot3(xyz(r2), wro) + r2.w);
            lrd = mk(dot3(xyz(r0), wrd), dot3(xyz(r1), wrd), dot3(xyz(r2), wrd));
            dSign = __ldg(&S.inst[4 * slot + 3].z);
            lslot = slot;
            ++vis.inst;
        }
        float t, det, u, v;
        uint32_t hb;
        ++vis.tri;
        if (!tri_hit(S, tri, lro, lrd, tmax, t, det, u, v, hb)) continue;
        if (ANY) {
            if ((hb & TB_SHADOW_OK) && side_ok(hb, det * dSign)) return true;
        } else if (side_ok(hb, det * dSign) && (hb & TB_CLOSEST_OK)) {
            tmax = t;
            bestTri = (int)tri;
            bestInst = (int)slot;
            bu = u;
            bv = v;
        }
    }
    return false;
}

// `sWide` holds the first `nWide` nodes of the tree (the top levels: nodes are
// numbered breadth-first) staged in shared memory, or nWide == 0.
template <bool ANY>
__device__ __forceinline__ bool wide_walk(const DevScene& S, float3 wro, float3 wrd, float& tmax, int& bestTri,
                                          int& bestInst, float& bu, float& bv, Visits& vis, uint32_t* err,
                                          const uint4* sWide = nullptr, uint32_t nWide = 0) {
    const float3 winv = mk(1.0f / wrd.x, 1.0f / wrd.y, 1.0f / wrd.z);
    if (SB_DYN_FIRST && dyn_walk<ANY>(S, wro, wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    // Box tests use the inverse clamped to +-1e30. An infinite one (a zero
    // direction component) would give q * inf = NaN for every child plane at
    // q = 0 and pass that axis for all of them: axis-parallel rays then visit
    // about 25x the nodes. Clamped, the plane distances stay finite and
    // signed, so the test still only keeps boxes the ray can reach.
    const float3 binv = mk(fminf(fmaxf(winv.x, -1e30f), 1e30f), fminf(fmaxf(winv.y, -1e30f), 1e30f),
                           fminf(fmaxf(winv.z, -1e30f), 1e30f));
    const uint32_t oct = (binv.x < 0.0f ? 1u : 0u) | (binv.y < 0.0f ? 2u : 0u) | (binv.z < 0.0f ? 4u : 0u);
    uint2 stk[SB_STACK];
    int sp = 0;
    uint32_t node = 0;  // the root (the wide tree is only built when non-empty)
    uint32_t gBase = 0, gBits = 0;  // interior hits << 24 | imask << 16
    uint32_t tBase = 0, tBits = 0;  // item hits
    uint32_t lslot = FLAT_NONE;
    float3 lro = wro, lrd = wrd;
    float dSign = 1.0f;
    uint32_t iter = 0;
    for (;;) {
        bool done = false;
        // node phase: until this lane holds items to test or has nothing left
        for (;;) {
            if (node == FLAT_NONE) {
                if (gBits >> 24) {
                    const uint32_t key = __ffs(gBits >> 24) - 1u;
                    gBits &= ~(1u << (24u + key));
                    const uint32_t slot = key ^ oct;
                    node = gBase + __popc((gBits >> 16) & 0xFFu & ((1u << slot) - 1u));
                    if (gBits >> 24) {
                        if (sp >= SB_STACK) {  // unreachable: the tree's depth was checked on build
                            latch(err, ERR_CAPACITY);
                            done = true;
                            break;
                        }
                        stk[sp++] = make_uint2(gBase, gBits);
                    }
                    gBits = 0;
                } else if (sp > 0) {
                    --sp;
                    gBase = stk[sp].x;
                    gBits = stk[sp].y;
                    continue;
                } else {
                    done = true;
                    break;
                }
            }
            if (++iter > S.iterCap) {
                latch(err, ERR_WATCHDOG);
                done = true;
                break;
            }
            wide_visit(S, node, wro, binv, oct, tmax, sWide, nWide, vis, gBase, gBits, tBase, tBits);
            node = FLAT_NONE;
            if (tBits) break;
        }
        if (done) break;
        // leaf phase (warp-aligned): items in slot order share the local ray
        if (wide_items<ANY>(S, tBase, tBits, wro, wrd, lslot, lro, lrd, dSign, tmax, bestTri, bestInst, bu, bv, vis))
            return true;
    }
    if (!SB_DYN_FIRST && dyn_walk<ANY>(S, wro, wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    return ANY ? false : bestTri >= 0;
}

// The same walk held between rounds (wide_begin, wide_step, wide_end), so that
// a persistent warp can give a lane a new ray as soon as its walk ends (the
// closest-hit stage's per-lane refill). Only that caller uses it: wide_walk
// keeps its state in registers, which a held walk cannot.
struct WideWalk {
    float3 wro, wrd, binv;
    uint32_t oct;
    uint32_t node;          // next node to visit, or FLAT_NONE
    uint32_t gBase, gBits;  // the group of hit interior children being visited
    uint32_t lslot;         // slot of the cached local ray
    float3 lro, lrd;
    float dSign;
    uint32_t iter;
    int sp;
    uint2 stk[SB_STACK];
};

// The moved slots first (SB_DYN_FIRST) and the walk's start. True: an any hit
// among the moved slots (the walk is over).
template <bool ANY>
__device__ __forceinline__ bool wide_begin(const DevScene& S, WideWalk& w, float3 wro, float3 wrd, float& tmax,
                                           int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                           uint32_t* err) {
    const float3 winv = mk(1.0f / wrd.x, 1.0f / wrd.y, 1.0f / wrd.z);
    if (SB_DYN_FIRST && dyn_walk<ANY>(S, wro, wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    // the inverse clamped to +-1e30, as in wide_walk
    w.binv = mk(fminf(fmaxf(winv.x, -1e30f), 1e30f), fminf(fmaxf(winv.y, -1e30f), 1e30f),
                fminf(fmaxf(winv.z, -1e30f), 1e30f));
    w.oct = (w.binv.x < 0.0f ? 1u : 0u) | (w.binv.y < 0.0f ? 2u : 0u) | (w.binv.z < 0.0f ? 4u : 0u);
    w.wro = wro;
    w.wrd = wrd;
    w.sp = 0;
    w.node = 0;  // the root (the wide tree is only built when non-empty)
    w.gBase = 0;
    w.gBits = 0;
    w.lslot = FLAT_NONE;
    w.lro = wro;
    w.lrd = wrd;
    w.dSign = 1.0f;
    w.iter = 0;
    return false;
}

// After the tree: the moved slots when they go last, and the walk's result.
template <bool ANY>
__device__ __forceinline__ bool wide_end(const DevScene& S, const WideWalk& w, float& tmax, int& bestTri,
                                         int& bestInst, float& bu, float& bv, Visits& vis, uint32_t* err) {
    if (!SB_DYN_FIRST) {
        const float3 winv = mk(1.0f / w.wrd.x, 1.0f / w.wrd.y, 1.0f / w.wrd.z);
        if (dyn_walk<ANY>(S, w.wro, w.wrd, winv, tmax, bestTri, bestInst, bu, bv, vis, err)) return true;
    }
    return ANY ? false : bestTri >= 0;
}

// One round: nodes until this lane holds items to test (or has nothing left),
// then those items. Returns 0 to go on, 1 when the tree is done (or a capacity
// / watchdog error ended it), 2 on an any hit.
//
// sStack, when given, holds the group stack in shared memory instead: this
// thread's column of a [entry][thread] array (entry e at sStack[e * blockDim.x],
// so the lanes of a warp use distinct banks whatever their stack depths), with
// room for sDepth entries.
template <bool ANY>
__device__ __forceinline__ int wide_step(const DevScene& S, WideWalk& w, float& tmax, int& bestTri, int& bestInst,
                                         float& bu, float& bv, Visits& vis, uint32_t* err,
                                         const uint4* sWide = nullptr, uint32_t nWide = 0, uint2* sStack = nullptr,
                                         int sDepth = 0) {
    uint32_t tBase = 0, tBits = 0;
    for (;;) {
        if (w.node == FLAT_NONE) {
            if (w.gBits >> 24) {
                const uint32_t key = __ffs(w.gBits >> 24) - 1u;
                w.gBits &= ~(1u << (24u + key));
                const uint32_t slot = key ^ w.oct;
                w.node = w.gBase + __popc((w.gBits >> 16) & 0xFFu & ((1u << slot) - 1u));
                if (w.gBits >> 24) {
                    if (w.sp >= (sStack ? sDepth : SB_STACK)) {  // unreachable: the depth was checked
                        latch(err, ERR_CAPACITY);
                        return 1;
                    }
                    if (sStack) sStack[(uint32_t)w.sp * blockDim.x] = make_uint2(w.gBase, w.gBits);
                    else w.stk[w.sp] = make_uint2(w.gBase, w.gBits);
                    ++w.sp;
                }
                w.gBits = 0;
            } else if (w.sp > 0) {
                --w.sp;
                const uint2 e = sStack ? sStack[(uint32_t)w.sp * blockDim.x] : w.stk[w.sp];
                w.gBase = e.x;
                w.gBits = e.y;
                continue;
            } else {
                return 1;
            }
        }
        if (++w.iter > S.iterCap) {
            latch(err, ERR_WATCHDOG);
            return 1;
        }
        wide_visit(S, w.node, w.wro, w.binv, w.oct, tmax, sWide, nWide, vis, w.gBase, w.gBits, tBase, tBits);
        w.node = FLAT_NONE;
        if (tBits) break;
    }
    return wide_items<ANY>(S, tBase, tBits, w.wro, w.wrd, w.lslot, w.lro, w.lrd, w.dSign, tmax, bestTri, bestInst, bu,
                           bv, vis)
               ? 2
               : 0;
}

// Traversal schedule per query kind: 0 nested (as the reference), 1 unified
// two-level loop, 2 nested with while-while BLAS walks. Measured on the
// 262k-triangle atrium (B200): closest hit 0.51 / 0.41 / 0.57 ms, any hit
// 0.35 / 0.80 / 0.54 ms for 0 / 1 / 2 — hence the defaults.
#ifndef SB_CLOSEST_WALK
#define SB_CLOSEST_WALK 1
#endif
#ifndef SB_ANY_WALK
#define SB_ANY_WALK 0
#endif
// Child-pair walk per query kind when the pair layout is usable. Measured on
// the atrium: closest hit 0.413 -> 0.374 ms with pairs; any hit 0.353 (nested,
// stackless) -> 0.665 ms with pairs, so any hit keeps the nested walk.
#ifndef SB_CLOSEST_PAIRS
#define SB_CLOSEST_PAIRS 1
#endif
#ifndef SB_ANY_PAIRS
#define SB_ANY_PAIRS 0
#endif
__device__ __forceinline__ bool closest_pairs(const DevScene& S) { return SB_CLOSEST_PAIRS && pairs_usable(S); }
__device__ __forceinline__ bool any_pairs(const DevScene& S) { return SB_ANY_PAIRS && pairs_usable(S); }

// traverseClosest, spectral_traverse.js:441-474. With `pairs` (pairs_usable),
// `tl` is the TLAS child-pair array, else the 32-byte TLAS nodes. On the
// 8-wide scene BVH, `sWide` / `nWide` are its staged top nodes (wide_walk).
__device__ __forceinline__ void trace_closest(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float& bestT,
                                              int& bestTri, int& bestInst, float& bu, float& bv, Visits& vis,
                                              uint32_t* err, bool pairs, const uint4* sWide = nullptr,
                                              uint32_t nWide = 0) {
    bestT = T_MAX;
    bestTri = -1;
    bestInst = -1;
    bu = bv = 0.0f;
    if (S.wideNodes) {
        wide_walk<false>(S, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err, sWide, nWide);
        return;
    }
    if (S.flatOn) {
        flat_walk<false>(S, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err);
        return;
    }
    if (pairs) {
        pair_walk<false>(S, tl, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err);
        return;
    }
#if SB_CLOSEST_WALK == 1
    walk<false>(S, tl, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err);
#else
    nested_walk<false, SB_CLOSEST_WALK == 2>(S, tl, ro, rd, bestT, bestTri, bestInst, bu, bv, vis, err);
#endif
}

// traverseAny, spectral_traverse.js:539-569 (`tl` as for trace_closest)
__device__ __forceinline__ bool trace_any(const DevScene& S, const uint4* tl, float3 ro, float3 rd, float maxDist,
                                          Visits& vis, uint32_t* err, bool pairs) {
    int tri = -1, inst = -1;
    float u = 0.f, v = 0.f;
    if (S.flatOn) return flat_walk<true>(S, ro, rd, maxDist, tri, inst, u, v, vis, err);
    if (pairs) return pair_walk<true>(S, tl, ro, rd, maxDist, tri, inst, u, v, vis, err);
#if SB_ANY_WALK == 1
    return walk<true>(S, tl, ro, rd, maxDist, tri, inst, u, v, vis, err);
#else
    return nested_walk<true, SB_ANY_WALK == 2>(S, tl, ro, rd, maxDist, tri, inst, u, v, vis, err);
#endif
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

// sampleAtlas, gi_probes.js:1941-1974: 8-tap trilinear over the cage probes,
// each tap a bilinear fetch of the previous RGBA16F atlas (exact weights; the
// 2x2 footprint stays inside the probe's tile, so no edge clamp applies).
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
    // the bilinear footprint inside each cage probe's tile: tile-local coordinate
    // 0.5 + uv * 6 in [0.5, 6.5], the same offset and weights for all 8 taps
    const float2 ouv = oct_encode(normalize3(N));
    const float xl = fmaf(ouv.x, 6.0f, 0.5f), yl = fmaf(ouv.y, 6.0f, 0.5f);
    const float fx0 = floorf(xl), fy0 = floorf(yl), fx = xl - fx0, fy = yl - fy0;
    const uint32_t Wu = C.atlasW, off = (uint32_t)fy0 * Wu + (uint32_t)fx0;
    const float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy), w01 = (1.0f - fx) * fy, w11 = fx * fy;
    float3 acc = mk(0.f, 0.f, 0.f);
    float wsum = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        float px = base[0] + float(dx), py = base[1] + float(dy), pz = base[2] + float(dz);
        float wx = dx ? frac[0] : 1.0f - frac[0];
        float wy = dy ? frac[1] : 1.0f - frac[1];
        float wz = dz ? frac[2] : 1.0f - frac[2];
        float w = wx * wy * wz + 1e-4f;
        const uint32_t tile = ((uint32_t)pz * C.res[1] + (uint32_t)py) * 8u * Wu + (uint32_t)px * 8u;
        const uint2* p = C.atlasPrev + tile + off;
        float4 t00 = half4_to_float4(__ldg(p)), t10 = half4_to_float4(__ldg(p + 1));
        float4 t01 = half4_to_float4(__ldg(p + Wu)), t11 = half4_to_float4(__ldg(p + Wu + 1));
        float3 s = mk(t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11,
                      t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11,
                      t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11);
        acc = acc + s * w;
        wsum += w;
    }
    return acc * (1.0f / fmaxf(wsum, 1e-4f));
}

}  // namespace sb
