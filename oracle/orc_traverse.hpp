// orc_traverse.hpp — restatement of the two-level stackless traversal
// (spectral_traverse.js:116-569) over the reference's pooled layouts.
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
#pragma once
#include "orc_core.hpp"

namespace orc {

// The typed arrays buildSpectralScene returns (spectral_scene.js:2011-2033).
struct Scene {
    const uint32_t* nodes = nullptr;  // 8 u32 per node (spectral_scene.js:1225-1234)
    uint32_t nodeCount = 0;
    const uint32_t* triIndex = nullptr;
    uint32_t triCount = 0;
    const float* vertexData = nullptr;  // 8 f32 per vertex, LOCAL space
    uint32_t vertexCount = 0;
    const uint32_t* triMaterial = nullptr;
    const float* materials = nullptr;  // ubers | instances | TLAS (spectral_scene.js:1327-1334)
    uint32_t materialsLen = 0;
    uint32_t instBase = 0, instCount = 0, tlasBase = 0, tlasNodeCount = 0;
};

inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// Per-ray work counters (feed the bytes-per-ray model).
struct Counters {
    uint64_t tlasNodes = 0, instances = 0, blasNodes = 0, triTests = 0;
    void add(const Counters& o) {
        tlasNodes += o.tlasNodes; instances += o.instances; blasNodes += o.blasNodes; triTests += o.triTests;
    }
};

template <class R> struct Traverser {
    const Scene& s;
    Counters* cnt = nullptr;
    bool track2 = false;  // also track the second-nearest accepted t (widens the cull)
    explicit Traverser(const Scene& sc) : s(sc) {}

    // accessors, spectral_traverse.js:122-165
    V3<R> fetch_vert(uint32_t vid) const {
        const float* v = s.vertexData + (size_t)vid * VSTRIDE;
        return {R(v[0]), R(v[1]), R(v[2])};
    }
    uint32_t tri_vert(uint32_t tri, int k) const { return s.triIndex[(size_t)tri * 3 + k]; }
    R mat_f(uint32_t m, int k) const { return R(s.materials[(size_t)m * MAT_STRIDE + k]); }
    R inst_f(uint32_t i, int k) const { return R(s.materials[s.instBase + (size_t)i * INST_STRIDE + k]); }
    V3<R> inst_row(uint32_t i, int r) const { return {inst_f(i, r * 4), inst_f(i, r * 4 + 1), inst_f(i, r * 4 + 2)}; }
    V3<R> inst_inv_point(uint32_t i, V3<R> p) const {
        return {dot(inst_row(i, 0), p) + inst_f(i, 3), dot(inst_row(i, 1), p) + inst_f(i, 7),
                dot(inst_row(i, 2), p) + inst_f(i, 11)};
    }
    V3<R> inst_inv_dir(uint32_t i, V3<R> d) const {
        return {dot(inst_row(i, 0), d), dot(inst_row(i, 1), d), dot(inst_row(i, 2), d)};
    }
    // (M^-1)^T n, spectral_traverse.js:155-156
    V3<R> inst_normal_to_world(uint32_t i, V3<R> n) const {
        return normalize(inst_row(i, 0) * n.x + inst_row(i, 1) * n.y + inst_row(i, 2) * n.z);
    }
    R tlas_f(uint32_t n, int k) const { return R(s.materials[s.tlasBase + (size_t)n * TLAS_STRIDE + k]); }

    // spectral_traverse.js:193-202
    bool side_accepts(uint32_t m, R det) const {
        R side = mat_f(m, 22);
        bool front = det > R(0);
        return side >= R(1.5) || (side < R(0.5) && front) ||
               (side >= R(0.5) && side < R(1.5) && det < R(0));
    }
    // spectral_traverse.js:204-220 with no map bound (the untextured path: the
    // alpha comes from the constant opacity in slot 10).
    bool alpha_accepts(uint32_t m) const {
        R alpha = mat_f(m, 10);
        R alphaTest = mat_f(m, 23);
        return alpha > R(1.0e-4) && (alphaTest <= R(0) || alpha >= alphaTest);
    }
    uint32_t flags(uint32_t m) const { return (uint32_t)mat_f(m, 26); }

    // Möller–Trumbore as written at spectral_traverse.js:393-409.
    // Returns true and (t, det, u, v) when the triangle is hit in (RAY_EPS, tmax).
    bool mt(uint32_t tri, V3<R> ro, V3<R> rd, R tmax, R& t, R& det, R& u, R& vb) const {
        V3<R> p0 = fetch_vert(tri_vert(tri, 0)), p1 = fetch_vert(tri_vert(tri, 1)), p2 = fetch_vert(tri_vert(tri, 2));
        V3<R> e1 = p1 - p0, e2 = p2 - p0;
        V3<R> pv = cross(rd, e2);
        det = dot(e1, pv);
        if (!(std::fabs(det) > R(1e-12))) return false;
        R invDet = R(1) / det;
        V3<R> tv = ro - p0;
        u = dot(tv, pv) * invDet;
        if (!(u >= R(0) && u <= R(1))) return false;
        V3<R> qv = cross(tv, e1);
        vb = dot(rd, qv) * invDet;
        if (!(vb >= R(0) && u + vb <= R(1))) return false;
        t = dot(e2, qv) * invDet;
        return t > R(RAY_EPS) && t < tmax;
    }

    // slab test, spectral_traverse.js:375-382
    static bool slab(const R bmin[3], const R bmax[3], V3<R> ro, V3<R> invD, R tlimit) {
        R t0x = (bmin[0] - ro.x) * invD.x, t1x = (bmax[0] - ro.x) * invD.x;
        R t0y = (bmin[1] - ro.y) * invD.y, t1y = (bmax[1] - ro.y) * invD.y;
        R t0z = (bmin[2] - ro.z) * invD.z, t1z = (bmax[2] - ro.z) * invD.z;
        // WGSL min/max of a NaN operand are implementation-defined; the IEEE-754
        // minNum/maxNum reading (NaN ignored) is used here and on the GPU.
        R tNear = std::fmax(std::fmax(std::fmin(t0x, t1x), std::fmin(t0y, t1y)), std::fmin(t0z, t1z));
        R tFar = std::fmin(std::fmin(std::fmax(t0x, t1x), std::fmax(t0y, t1y)), std::fmax(t0z, t1z));
        return tFar >= std::fmax(tNear, R(0)) && tNear < tlimit;
    }

    // blasClosest, spectral_traverse.js:354-435. Also tracks the second-nearest
    // accepted candidate t (near-tie exemption of the hit-ID parity rule).
    void blas_closest(uint32_t inst, V3<R> wro, V3<R> wrd, R& bestT, int& bestTri, int& bestInst,
                      R& secondT) const {
        V3<R> ro = inst_inv_point(inst, wro), rd = inst_inv_dir(inst, wrd);
        R dSign = inst_f(inst, 14);
        V3<R> invD(R(1) / rd.x, R(1) / rd.y, R(1) / rd.z);
        uint32_t blasEnd = (uint32_t)inst_f(inst, 13);
        uint32_t cursor = (uint32_t)inst_f(inst, 12);
        for (uint32_t it = 0; it < s.nodeCount; ++it) {
            if (cursor >= blasEnd) break;
            const uint32_t* nd = s.nodes + (size_t)cursor * 8;
            R bmin[3] = {R(u2f(nd[0])), R(u2f(nd[1])), R(u2f(nd[2]))};
            R bmax[3] = {R(u2f(nd[3])), R(u2f(nd[4])), R(u2f(nd[5]))};
            uint32_t miss = nd[6], payload = nd[7];
            if (cnt) cnt->blasNodes++;
            // With track2 the cull uses secondT (>= bestT) so candidates behind the
            // best are seen too; bestT/bestTri are unchanged by the wider cull.
            if (slab(bmin, bmax, ro, invD, track2 ? secondT : bestT)) {
                if (payload == 0xFFFFFFFFu) {
                    cursor = cursor + 1;
                } else {
                    uint32_t triOffset = payload & 0x00FFFFFFu, triCount = payload >> 24;
                    for (uint32_t i = 0; i < triCount; ++i) {
                        uint32_t tri = triOffset + i;
                        if (cnt) cnt->triTests++;
                        R t, det, u, vb;
                        if (!mt(tri, ro, rd, track2 ? secondT : bestT, t, det, u, vb)) continue;
                        uint32_t m = s.triMaterial[tri];
                        uint32_t fl = flags(m);
                        bool acc = side_accepts(m, det * dSign) && ((fl & 1u) ? alpha_accepts(m) : (fl & 2u) != 0);
                        if (!acc) continue;
                        if (t < bestT) {
                            secondT = bestT;
                            bestT = t;
                            bestTri = (int)tri;
                            bestInst = (int)inst;
                        } else if (t < secondT) {
                            secondT = t;
                        }
                    }
                    cursor = miss;
                }
            } else {
                cursor = miss;
            }
        }
    }

    // traverseClosest, spectral_traverse.js:441-474
    void closest(V3<R> ro, V3<R> rd, R& bestT, int& bestTri, int& bestInst, R& secondT) const {
        bestT = R(T_MAX);
        secondT = R(T_MAX);
        bestTri = -1;
        bestInst = -1;
        V3<R> invD(R(1) / rd.x, R(1) / rd.y, R(1) / rd.z);
        uint32_t cursor = 0;
        for (uint32_t it = 0; it < s.tlasNodeCount; ++it) {
            if (cursor >= s.tlasNodeCount) break;
            R bmin[3] = {tlas_f(cursor, 0), tlas_f(cursor, 1), tlas_f(cursor, 2)};
            R bmax[3] = {tlas_f(cursor, 3), tlas_f(cursor, 4), tlas_f(cursor, 5)};
            uint32_t miss = (uint32_t)tlas_f(cursor, 6);
            R instCountF = tlas_f(cursor, 8);
            if (cnt) cnt->tlasNodes++;
            if (slab(bmin, bmax, ro, invD, track2 ? secondT : bestT)) {
                if (instCountF < R(0.5)) {
                    cursor = cursor + 1;
                } else {
                    uint32_t off = (uint32_t)tlas_f(cursor, 7);
                    for (uint32_t i = 0; i < (uint32_t)instCountF; ++i) {
                        uint32_t inst = off + i;
                        if (cnt) cnt->instances++;
                        if (inst_f(inst, 15) > R(0.5)) blas_closest(inst, ro, rd, bestT, bestTri, bestInst, secondT);
                    }
                    cursor = miss;
                }
            } else {
                cursor = miss;
            }
        }
    }

    // blasAny, spectral_traverse.js:477-536
    void blas_any(uint32_t inst, V3<R> wro, V3<R> wrd, R maxDist, bool& blocked) const {
        V3<R> ro = inst_inv_point(inst, wro), rd = inst_inv_dir(inst, wrd);
        R dSign = inst_f(inst, 14);
        V3<R> invD(R(1) / rd.x, R(1) / rd.y, R(1) / rd.z);
        uint32_t blasEnd = (uint32_t)inst_f(inst, 13);
        uint32_t cursor = (uint32_t)inst_f(inst, 12);
        for (uint32_t it = 0; it < s.nodeCount; ++it) {
            if (cursor >= blasEnd || blocked) break;
            const uint32_t* nd = s.nodes + (size_t)cursor * 8;
            R bmin[3] = {R(u2f(nd[0])), R(u2f(nd[1])), R(u2f(nd[2]))};
            R bmax[3] = {R(u2f(nd[3])), R(u2f(nd[4])), R(u2f(nd[5]))};
            uint32_t miss = nd[6], payload = nd[7];
            if (cnt) cnt->blasNodes++;
            if (slab(bmin, bmax, ro, invD, maxDist)) {
                if (payload == 0xFFFFFFFFu) {
                    cursor = cursor + 1;
                } else {
                    uint32_t triOffset = payload & 0x00FFFFFFu, triCount = payload >> 24;
                    for (uint32_t i = 0; i < triCount; ++i) {
                        uint32_t tri = triOffset + i;
                        if (cnt) cnt->triTests++;
                        R t, det, u, vb;
                        if (!mt(tri, ro, rd, maxDist, t, det, u, vb)) continue;
                        uint32_t m = s.triMaterial[tri];
                        uint32_t fl = flags(m);
                        if (side_accepts(m, det * dSign) && (fl & 4u)) {
                            if ((fl & 1u) ? alpha_accepts(m) : (fl & 2u) != 0) blocked = true;
                        }
                    }
                    cursor = miss;
                }
            } else {
                cursor = miss;
            }
        }
    }

    // traverseAny, spectral_traverse.js:539-569
    bool any(V3<R> ro, V3<R> rd, R maxDist) const {
        V3<R> invD(R(1) / rd.x, R(1) / rd.y, R(1) / rd.z);
        uint32_t cursor = 0;
        bool blocked = false;
        for (uint32_t it = 0; it < s.tlasNodeCount; ++it) {
            if (cursor >= s.tlasNodeCount || blocked) break;
            R bmin[3] = {tlas_f(cursor, 0), tlas_f(cursor, 1), tlas_f(cursor, 2)};
            R bmax[3] = {tlas_f(cursor, 3), tlas_f(cursor, 4), tlas_f(cursor, 5)};
            uint32_t miss = (uint32_t)tlas_f(cursor, 6);
            R instCountF = tlas_f(cursor, 8);
            if (cnt) cnt->tlasNodes++;
            if (slab(bmin, bmax, ro, invD, maxDist)) {
                if (instCountF < R(0.5)) {
                    cursor = cursor + 1;
                } else {
                    uint32_t off = (uint32_t)tlas_f(cursor, 7);
                    for (uint32_t i = 0; i < (uint32_t)instCountF; ++i) {
                        uint32_t inst = off + i;
                        if (cnt) cnt->instances++;
                        if (inst_f(inst, 15) > R(0.5)) blas_any(inst, ro, rd, maxDist, blocked);
                    }
                    cursor = miss;
                }
            } else {
                cursor = miss;
            }
        }
        return blocked;
    }

    // Independent cross-check: closest accepted hit over every triangle of every
    // active instance, no BVH involved.
    void brute_closest(V3<R> ro, V3<R> rd, R& bestT, int& bestTri, int& bestInst) const {
        bestT = R(T_MAX);
        bestTri = -1;
        bestInst = -1;
        for (uint32_t inst = 0; inst < s.instCount; ++inst) {
            if (!(inst_f(inst, 15) > R(0.5))) continue;
            V3<R> lro = inst_inv_point(inst, ro), lrd = inst_inv_dir(inst, rd);
            R dSign = inst_f(inst, 14);
            uint32_t root = (uint32_t)inst_f(inst, 12), end = (uint32_t)inst_f(inst, 13);
            // the BLAS's triangles are those referenced by its leaves
            for (uint32_t n = root; n < end; ++n) {
                uint32_t payload = s.nodes[(size_t)n * 8 + 7];
                if (payload == 0xFFFFFFFFu) continue;
                uint32_t off = payload & 0x00FFFFFFu, c = payload >> 24;
                for (uint32_t i = 0; i < c; ++i) {
                    R t, det, u, vb;
                    uint32_t tri = off + i;
                    if (!mt(tri, lro, lrd, bestT, t, det, u, vb)) continue;
                    uint32_t m = s.triMaterial[tri];
                    uint32_t fl = flags(m);
                    if (side_accepts(m, det * dSign) && ((fl & 1u) ? alpha_accepts(m) : (fl & 2u) != 0)) {
                        bestT = t;
                        bestTri = (int)tri;
                        bestInst = (int)inst;
                    }
                }
            }
        }
    }
};

}  // namespace orc
