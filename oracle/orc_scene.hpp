// orc_scene.hpp — restatement of the refit and TLAS lanes:
//   gi_refit.js:34-165 (BLAS refit), 245-292 (TLAS range refit),
//   298-346 (TLAS refit index), 352-430 (sparse dirty refit);
//   spectral_scene.js:973-1003 (buildTlasRecords), 1256-1298 (computeDynamic),
//   1339-1366 (writeDynamic), 1402-1514 (updateTransforms).
// The three.js math the reference calls (Matrix4.invert / determinant,
// Box3.applyMatrix4; three r185, not vendored) is restated from the
// mathematics: inverse = adjugate / determinant with cofactors from 2x2
// minors, AABB = min/max over the 8 transformed corners. Its operation order
// against three itself is unpinned.
// TEST INFRASTRUCTURE ONLY (see orc_core.hpp).
#pragma once
#include "orc_core.hpp"
#include <limits>

namespace orc {

// JS Math.min / Math.max: NaN-propagating, -0 < +0.
inline float js_min(float a, float b) {
    if (std::isnan(a) || std::isnan(b)) return NAN;
    if (a == b) return std::signbit(a) ? a : b;
    return a < b ? a : b;
}
inline float js_max(float a, float b) {
    if (std::isnan(a) || std::isnan(b)) return NAN;
    if (a == b) return std::signbit(a) ? b : a;
    return a > b ? a : b;
}

// refitFlatBlasRange (gi_refit.js:158-165 over the stepper 34-156, run to
// completion). nodes is the u32 view; bounds are written through the f32 view.
inline bool refit_blas(uint32_t* nodes, size_t nodesLen, const uint32_t* triIndex, size_t triIndexLen,
                       const float* vertexData, size_t vertexDataLen, int64_t root, int64_t end) {
    if (!nodes || !triIndex || !vertexData || root < 0 || end <= root || (size_t)end * 8 > nodesLen) return false;
    auto F = [&](size_t i) -> float& { return *reinterpret_cast<float*>(&nodes[i]); };
    for (int64_t i = end - 1; i >= root; --i) {
        size_t base = (size_t)i * 8;
        uint32_t info = nodes[base + 7];
        if (info != 0xFFFFFFFFu) {
            uint32_t triOff = info & 0x00FFFFFFu, triCnt = info >> 24;
            if (triCnt == 0) continue;  // empty leaf keeps its stale bounds
            float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
            for (uint32_t t = triOff; t < triOff + triCnt; ++t) {
                size_t t3 = (size_t)t * 3;
                if (t3 + 2 >= triIndexLen) return false;
                for (int k = 0; k < 3; ++k) {
                    size_t dd = (size_t)triIndex[t3 + k] * 8;
                    if (dd + 2 >= vertexDataLen) return false;
                    float x = vertexData[dd], y = vertexData[dd + 1], z = vertexData[dd + 2];
                    if (x < mnx) mnx = x;
                    if (x > mxx) mxx = x;
                    if (y < mny) mny = y;
                    if (y > mxy) mxy = y;
                    if (z < mnz) mnz = z;
                    if (z > mxz) mxz = z;
                }
            }
            F(base) = mnx; F(base + 1) = mny; F(base + 2) = mnz;
            F(base + 3) = mxx; F(base + 4) = mxy; F(base + 5) = mxz;
        } else {
            int64_t l = i + 1;
            if (l >= end) return false;
            int64_t r = nodes[(size_t)l * 8 + 6];
            if (!(r > l && r < end)) return false;
            size_t lb = (size_t)l * 8, rb = (size_t)r * 8;
            F(base) = js_min(F(lb), F(rb));
            F(base + 1) = js_min(F(lb + 1), F(rb + 1));
            F(base + 2) = js_min(F(lb + 2), F(rb + 2));
            F(base + 3) = js_max(F(lb + 3), F(rb + 3));
            F(base + 4) = js_max(F(lb + 4), F(rb + 4));
            F(base + 5) = js_max(F(lb + 5), F(rb + 5));
        }
    }
    return true;
}

inline bool is_int(float v) { return std::isfinite(v) && std::floor(v) == v; }

// refitFlatTlasRange, gi_refit.js:245-292 (f32 TLAS view, f32 instance bounds).
inline bool refit_tlas_range(float* nodes, size_t nodesLen, const float* ib, size_t ibLen, int64_t root, int64_t end) {
    int64_t nodeEnd = end >= 0 ? end : (int64_t)(nodesLen / 12);
    int64_t instanceCount = (int64_t)(ibLen / 6);
    if (root < 0 || nodeEnd <= root || (size_t)nodeEnd * 12 > nodesLen) return false;
    for (int64_t i = nodeEnd - 1; i >= root; --i) {
        size_t base = (size_t)i * 12;
        float leafCount = nodes[base + 8];
        float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
        if (leafCount > 0) {
            float off = nodes[base + 7];
            if (!is_int(off) || !is_int(leafCount) || off < 0 || leafCount < 1 || off + leafCount > instanceCount) return false;
            for (int64_t slot = (int64_t)off; slot < (int64_t)off + (int64_t)leafCount; ++slot) {
                const float* b = ib + slot * 6;
                if (b[0] < mnx) mnx = b[0];
                if (b[1] < mny) mny = b[1];
                if (b[2] < mnz) mnz = b[2];
                if (b[3] > mxx) mxx = b[3];
                if (b[4] > mxy) mxy = b[4];
                if (b[5] > mxz) mxz = b[5];
            }
        } else {
            int64_t left = i + 1;
            if (left >= nodeEnd) return false;
            float right = nodes[(size_t)left * 12 + 6];
            if (!is_int(right) || !(right > left && right < nodeEnd)) return false;
            size_t lb = (size_t)left * 12, rb = (size_t)right * 12;
            mnx = js_min(nodes[lb], nodes[rb]);
            mny = js_min(nodes[lb + 1], nodes[rb + 1]);
            mnz = js_min(nodes[lb + 2], nodes[rb + 2]);
            mxx = js_max(nodes[lb + 3], nodes[rb + 3]);
            mxy = js_max(nodes[lb + 4], nodes[rb + 4]);
            mxz = js_max(nodes[lb + 5], nodes[rb + 5]);
        }
        nodes[base] = mnx; nodes[base + 1] = mny; nodes[base + 2] = mnz;
        nodes[base + 3] = mxx; nodes[base + 4] = mxy; nodes[base + 5] = mxz;
    }
    return true;
}

// createFlatTlasRefitIndex (gi_refit.js:298-346) + refitFlatTlasDirty (352-430).
// Returns the touched node list ascending, or false on a topology violation.
inline bool refit_tlas_dirty(float* nodes, size_t nodesLen, const float* ib, size_t ibLen, int64_t end,
                             const uint32_t* dirtySlots, size_t nDirty, std::vector<uint32_t>& touched) {
    int64_t nodeEnd = end;
    int64_t instanceCount = (int64_t)(ibLen / 6);
    if (nodeEnd <= 0 || (size_t)nodeEnd * 12 > nodesLen) return false;
    std::vector<int32_t> parent(nodeEnd, -1), leafBySlot(instanceCount, -1);
    for (int64_t i = 0; i < nodeEnd; ++i) {
        size_t base = (size_t)i * 12;
        float leafCount = nodes[base + 8];
        if (leafCount > 0) {
            float off = nodes[base + 7];
            if (!is_int(off) || !is_int(leafCount) || off < 0 || leafCount < 1 || off + leafCount > instanceCount) return false;
            for (int64_t s = (int64_t)off; s < (int64_t)off + (int64_t)leafCount; ++s) {
                if (leafBySlot[s] != -1) return false;
                leafBySlot[s] = (int32_t)i;
            }
        } else {
            int64_t left = i + 1;
            if (left >= nodeEnd) return false;
            float right = nodes[(size_t)left * 12 + 6];
            if (!is_int(right) || !(right > left && right < nodeEnd)) return false;
            if (parent[left] != -1 || parent[(int64_t)right] != -1) return false;
            parent[left] = (int32_t)i;
            parent[(int64_t)right] = (int32_t)i;
        }
    }
    for (int64_t s = 0; s < instanceCount; ++s) if (leafBySlot[s] < 0) return false;
    std::vector<char> mark(nodeEnd, 0);
    std::vector<uint32_t> dirty;
    for (size_t d = 0; d < nDirty; ++d) {
        int64_t slot = dirtySlots[d];
        if (slot < 0 || slot >= instanceCount) return false;
        int64_t node = leafBySlot[slot];
        while (node >= 0) {
            if (!mark[node]) { mark[node] = 1; dirty.push_back((uint32_t)node); }
            node = parent[node];
        }
    }
    std::sort(dirty.begin(), dirty.end(), std::greater<uint32_t>());
    for (uint32_t i : dirty) {
        size_t base = (size_t)i * 12;
        float leafCount = nodes[base + 8];
        float mnx = INFINITY, mny = INFINITY, mnz = INFINITY, mxx = -INFINITY, mxy = -INFINITY, mxz = -INFINITY;
        if (leafCount > 0) {
            int64_t off = (int64_t)nodes[base + 7];
            for (int64_t slot = off; slot < off + (int64_t)leafCount; ++slot) {
                const float* b = ib + slot * 6;
                if (b[0] < mnx) mnx = b[0];
                if (b[1] < mny) mny = b[1];
                if (b[2] < mnz) mnz = b[2];
                if (b[3] > mxx) mxx = b[3];
                if (b[4] > mxy) mxy = b[4];
                if (b[5] > mxz) mxz = b[5];
            }
        } else {
            size_t lb = (size_t)(i + 1) * 12, rb = (size_t)nodes[(size_t)(i + 1) * 12 + 6] * 12;
            mnx = js_min(nodes[lb], nodes[rb]);
            mny = js_min(nodes[lb + 1], nodes[rb + 1]);
            mnz = js_min(nodes[lb + 2], nodes[rb + 2]);
            mxx = js_max(nodes[lb + 3], nodes[rb + 3]);
            mxy = js_max(nodes[lb + 4], nodes[rb + 4]);
            mxz = js_max(nodes[lb + 5], nodes[rb + 5]);
        }
        nodes[base] = mnx; nodes[base + 1] = mny; nodes[base + 2] = mnz;
        nodes[base + 3] = mxx; nodes[base + 4] = mxy; nodes[base + 5] = mxz;
    }
    std::sort(dirty.begin(), dirty.end());
    touched = dirty;
    return true;
}

// ------------------------------------------------------------ instance math
// m: column-major 4x4 (three Matrix4.elements), element (row r, col c) = m[c*4+r].
struct Inv34 { double r[12]; };

// 4x4 determinant by cofactor expansion along the first column, using the
// 2x2 minors of rows 2..3 (pairs of columns).
inline double det4(const double* m) {
    auto a = [&](int r, int c) { return m[c * 4 + r]; };
    // 2x2 minors of rows 2,3
    double s01 = a(2, 0) * a(3, 1) - a(2, 1) * a(3, 0);
    double s02 = a(2, 0) * a(3, 2) - a(2, 2) * a(3, 0);
    double s03 = a(2, 0) * a(3, 3) - a(2, 3) * a(3, 0);
    double s12 = a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1);
    double s13 = a(2, 1) * a(3, 3) - a(2, 3) * a(3, 1);
    double s23 = a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2);
    // cofactors of row 0 via Laplace on rows (1) x minors(2,3)
    double c0 = a(1, 1) * s23 - a(1, 2) * s13 + a(1, 3) * s12;
    double c1 = a(1, 0) * s23 - a(1, 2) * s03 + a(1, 3) * s02;
    double c2 = a(1, 0) * s13 - a(1, 1) * s03 + a(1, 3) * s01;
    double c3 = a(1, 0) * s12 - a(1, 1) * s02 + a(1, 2) * s01;
    return a(0, 0) * c0 - a(0, 1) * c1 + a(0, 2) * c2 - a(0, 3) * c3;
}

// Inverse by the adjugate: inv(r,c) = cofactor(c,r) / det. Returns the first
// three rows (the reference stores rows 0..2 with w = translation,
// spectral_scene.js:1276-1282). A singular matrix yields zeros, as three's
// invert does.
inline void inverse_rows(const double* m, double out[12]) {
    auto a = [&](int r, int c) { return m[c * 4 + r]; };
    double det = det4(m);
    if (det == 0) { for (int i = 0; i < 12; ++i) out[i] = 0; return; }
    double inv = 1.0 / det;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) {
            // cofactor C(c, r): delete row c and column r of m
            int rows[3], cols[3];
            for (int i = 0, k = 0; i < 4; ++i) if (i != c) rows[k++] = i;
            for (int j = 0, k = 0; j < 4; ++j) if (j != r) cols[k++] = j;
            double m3 = a(rows[0], cols[0]) * (a(rows[1], cols[1]) * a(rows[2], cols[2]) - a(rows[1], cols[2]) * a(rows[2], cols[1]))
                      - a(rows[0], cols[1]) * (a(rows[1], cols[0]) * a(rows[2], cols[2]) - a(rows[1], cols[2]) * a(rows[2], cols[0]))
                      + a(rows[0], cols[2]) * (a(rows[1], cols[0]) * a(rows[2], cols[1]) - a(rows[1], cols[1]) * a(rows[2], cols[0]));
            double cof = ((r + c) & 1) ? -m3 : m3;
            out[r * 4 + c] = cof * inv;
        }
}

// World AABB of a local box under m: min/max over the 8 transformed corners
// (with the projective divide, which is exactly 1 for affine m).
inline void transform_box(const double* m, const double lmin[3], const double lmax[3], double wmin[3], double wmax[3]) {
    for (int a = 0; a < 3; ++a) { wmin[a] = INFINITY; wmax[a] = -INFINITY; }
    for (int i = 0; i < 8; ++i) {
        double x = (i & 1) ? lmax[0] : lmin[0];
        double y = (i & 2) ? lmax[1] : lmin[1];
        double z = (i & 4) ? lmax[2] : lmin[2];
        double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
        double p[3] = {(m[0] * x + m[4] * y + m[8] * z + m[12]) * w, (m[1] * x + m[5] * y + m[9] * z + m[13]) * w,
                       (m[2] * x + m[6] * y + m[10] * z + m[14]) * w};
        for (int a = 0; a < 3; ++a) {
            if (p[a] < wmin[a]) wmin[a] = p[a];
            if (p[a] > wmax[a]) wmax[a] = p[a];
        }
    }
}

struct Aabb { double mn[3], mx[3], c[3]; };

// computeDynamic's per-instance part (spectral_scene.js:1262-1294).
// lbounds: f32 local box per instance (6 per instance: min xyz, max xyz).
inline void compute_instance(const double* m, bool active, const float* lb, float invRowsOut[12], float& detSign, Aabb& box) {
    double inv[12];
    inverse_rows(m, inv);
    for (int i = 0; i < 12; ++i) invRowsOut[i] = (float)inv[i];
    detSign = det4(m) < 0 ? -1.0f : 1.0f;
    if (active) {
        double lmin[3] = {lb[0], lb[1], lb[2]}, lmax[3] = {lb[3], lb[4], lb[5]};
        transform_box(m, lmin, lmax, box.mn, box.mx);
    } else {
        for (int a = 0; a < 3; ++a) box.mn[a] = box.mx[a] = m[12 + a];
    }
    for (int a = 0; a < 3; ++a) box.c[a] = (box.mn[a] + box.mx[a]) * 0.5;
}

struct TlasRec { double bx[6]; bool leaf; uint32_t off, cnt, miss; };

// buildTlasRecords, spectral_scene.js:973-1003 (leafSize 2, stable sort).
inline void build_tlas(const std::vector<Aabb>& aabbs, std::vector<TlasRec>& recs, std::vector<uint32_t>& order,
                       uint32_t leafSize = 2) {
    order.resize(aabbs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (uint32_t)i;
    recs.clear();
    struct Frame { uint32_t lo, hi, idx, stage; };
    // iterative pre-order emulation of the recursive emit()
    std::vector<Frame> st;
    auto open = [&](uint32_t lo, uint32_t hi) -> uint32_t {
        TlasRec r;
        for (int k = 0; k < 3; ++k) { r.bx[k] = INFINITY; r.bx[3 + k] = -INFINITY; }
        r.leaf = false; r.off = r.cnt = r.miss = 0;
        for (uint32_t i = lo; i < hi; ++i) {
            const Aabb& a = aabbs[order[i]];
            for (int k = 0; k < 3; ++k) {
                if (a.mn[k] < r.bx[k]) r.bx[k] = a.mn[k];
                if (a.mx[k] > r.bx[3 + k]) r.bx[3 + k] = a.mx[k];
            }
        }
        recs.push_back(r);
        return (uint32_t)recs.size() - 1;
    };
    st.push_back({0, (uint32_t)order.size(), open(0, (uint32_t)order.size()), 0});
    while (!st.empty()) {
        Frame& f = st.back();
        TlasRec& r = recs[f.idx];
        uint32_t lo = f.lo, hi = f.hi;
        if (f.stage == 0) {
            if (hi - lo <= leafSize) {
                r.leaf = true; r.off = lo; r.cnt = hi - lo;
                r.miss = (uint32_t)recs.size();
                st.pop_back();
                continue;
            }
            double ex = r.bx[3] - r.bx[0], ey = r.bx[4] - r.bx[1], ez = r.bx[5] - r.bx[2];
            int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
            std::stable_sort(order.begin() + lo, order.begin() + hi,
                             [&](uint32_t a, uint32_t b) { return aabbs[a].c[axis] < aabbs[b].c[axis]; });
            f.stage = 1;
            uint32_t mid = (lo + hi) >> 1;
            uint32_t child = open(lo, mid);
            st.push_back({lo, mid, child, 0});
        } else if (f.stage == 1) {
            f.stage = 2;
            uint32_t mid = (lo + hi) >> 1;
            uint32_t child = open(mid, hi);
            st.push_back({mid, hi, child, 0});
        } else {
            r.miss = (uint32_t)recs.size();
            st.pop_back();
        }
    }
}

}  // namespace orc
