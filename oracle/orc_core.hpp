// orc_core.hpp — CPU restatement of the reference's DDGI probe-update math.
//
// TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA path, never the
// thing measured or shipped: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs load it. The product library
// (speedball_b200/csrc) shares no code with it.
//
// Parity status: UNPINNED against the reference itself. The reference is
// JavaScript + TSL/WGSL on WebGPU (no JS engine or WebGPU stack exists on
// either machine) and ships no golden vectors or tests for this path
// (its scripts/gi-oct-test.mjs and refit smoke tests are absent). This file is
// a line-by-line restatement of the cited reference code; its own known-answer
// tests live in tests/test_oracle_*.py.
//
// Everything is templated on the arithmetic type R: R = double is the FP64
// oracle the GPU is checked against; R = float is the FP32 CPU baseline.
// Reference citations are file:line within the speedball-gi 0.7.0 tree.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace orc {

// ---------------------------------------------------------------- constants
// gi_probes.js:53-56, 106, 122-123, 132-137, 176-190; spectral_traverse.js:34-35
constexpr int OCT_RES = 6, BORDER = 1, TILE = 8;
constexpr double PI = 3.141592653589793;
constexpr double T_MAX = 1e30, RAY_EPS = 1e-3;
constexpr double TRACE_SURFACE_BIAS_CELL = 0.005;
constexpr int MAX_LIGHTS = 64, LIGHT_STRIDE = 17, LIGHTS_PER_CELL = 16;
constexpr int LIGHT_CELL_STRIDE = LIGHTS_PER_CELL + 1, LIGHT_CELL_OVERFLOW = LIGHTS_PER_CELL + 1;
constexpr double GI_FILTER_K = 8.0, GI_FILTER_EPS = 0.001, GI_FILTER_REL = 0.0225;
constexpr int MAT_STRIDE = 28, INST_STRIDE = 28, TLAS_STRIDE = 12, VSTRIDE = 8;
inline double golden_angle() { return PI * (3.0 - std::sqrt(5.0)); }  // gi_probes.js:106

template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> mulv(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) {
    R l = length(a);
    return a * (R(1) / l);
}
template <class R> inline R clampv(R v, R lo, R hi) { return std::min(std::max(v, lo), hi); }
template <class R> inline R mixv(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> inline V3<R> mix3(V3<R> a, V3<R> b, R t) {
    return {mixv(a.x, b.x, t), mixv(a.y, b.y, t), mixv(a.z, b.z, t)};
}
template <class R> inline R luma(V3<R> c) { return c.x * R(0.2126) + c.y * R(0.7152) + c.z * R(0.0722); }

// ------------------------------------------------------------- binary16
// IEEE 754 binary16 round-to-nearest-even from a double, written from the
// format's definition (1 sign, 5 exponent, 10 fraction bits; bias 15). The
// WebGPU RGBA16F StorageTexture rounds the same way on textureStore.
inline uint16_t to_half(double v) {
    uint16_t sign = std::signbit(v) ? 0x8000 : 0;
    double a = std::fabs(v);
    if (std::isnan(v)) return 0x7E00;
    if (a >= 65520.0) return sign | 0x7C00;  // rounds to infinity
    if (a < std::ldexp(1.0, -25)) return sign;  // below half the smallest subnormal (ties to 0 handled next)
    int e;
    std::frexp(a, &e);  // a = m * 2^e, m in [0.5,1)
    int exp = e - 1;    // a = 1.f * 2^exp
    if (exp < -14) {
        // subnormal: quantum 2^-24
        double q = a / std::ldexp(1.0, -24);
        double r = std::nearbyint(q);  // default rounding mode: nearest-even
        return sign | (uint16_t)r;     // r may reach 1024 = smallest normal, encoded correctly
    }
    double q = a / std::ldexp(1.0, exp - 10);  // in [1024, 2048)
    double r = std::nearbyint(q);
    int ex = exp;
    if (r >= 2048.0) { r = 1024.0; ex += 1; }
    if (ex > 15) return sign | 0x7C00;
    return sign | (uint16_t)((ex + 15) << 10) | (uint16_t)((int)r - 1024);
}
inline double from_half(uint16_t h) {
    int s = h >> 15, e = (h >> 10) & 31, f = h & 1023;
    double v;
    if (e == 0) v = std::ldexp((double)f, -24);
    else if (e == 31) v = f ? NAN : INFINITY;
    else v = std::ldexp(1024.0 + f, e - 25);
    return s ? -v : v;
}

// ----------------------------------------------------------- octahedral map
// gi_oct.js:25-40 (octEncode; the TSL twin 61-73 uses max(l1, 1e-20))
template <class R> inline void oct_encode(V3<R> n, R& u, R& v) {
    R l1 = std::fabs(n.x) + std::fabs(n.y) + std::fabs(n.z);
    R inv = R(1) / std::max(l1, R(1e-20));
    R ox = n.x * inv, oy = n.y * inv;
    if (n.z < R(0)) {
        R fx = (R(1) - std::fabs(oy)) * (ox >= R(0) ? R(1) : R(-1));
        R fy = (R(1) - std::fabs(ox)) * (oy >= R(0) ? R(1) : R(-1));
        ox = fx;
        oy = fy;
    }
    u = ox * R(0.5) + R(0.5);
    v = oy * R(0.5) + R(0.5);
}
// gi_oct.js:43-57 / 76-85
template <class R> inline V3<R> oct_decode(R u, R v) {
    R fx = u * R(2) - R(1), fy = v * R(2) - R(1);
    R nz = R(1) - std::fabs(fx) - std::fabs(fy);
    R t = std::max(-nz, R(0));
    R nx = fx + (fx >= R(0) ? -t : t);
    R ny = fy + (fy >= R(0) ? -t : t);
    return normalize(V3<R>(nx, ny, nz));
}

// ---------------------------------------------------------------- grid
struct Grid {
    double gridMin[3], gridSize[3];
    uint32_t res[3];
    uint32_t rays;
    double maxDist, cellMin;
    uint32_t probeTotal() const { return res[0] * res[1] * res[2]; }
    uint32_t atlasW() const { return res[0] * TILE; }
    uint32_t atlasH() const { return res[1] * res[2] * TILE; }
};

// gi_probes.js:1714-1726 (probeWorldPos); relocation offset * classifyStrength
// (probeTraceOrigin 1876-1885) is zero because classification is inert
// (classifyStrength defaults to 0, gi_probes.js:1215).
template <class R> inline V3<R> probe_world_pos(const Grid& g, uint32_t p) {
    uint32_t ix = p % g.res[0], iy = (p / g.res[0]) % g.res[1], iz = p / (g.res[0] * g.res[1]);
    R fx = R(ix) / std::max(R(1), R(g.res[0]) - R(1));
    R fy = R(iy) / std::max(R(1), R(g.res[1]) - R(1));
    R fz = R(iz) / std::max(R(1), R(g.res[2]) - R(1));
    return {R(g.gridMin[0]) + fx * R(g.gridSize[0]), R(g.gridMin[1]) + fy * R(g.gridSize[1]),
            R(g.gridMin[2]) + fz * R(g.gridSize[2])};
}

// gi_probes.js:1692-1704 (rayDir), normalized by every caller (1984, 2331).
template <class R> inline V3<R> ray_dir(uint32_t k, uint32_t rays, R jitter) {
    R sk = (R(k) + R(0.5)) / R(rays);
    R u = sk + jitter;
    R uw = u - std::floor(u);
    R z = R(1) - uw * R(2);
    R r = std::sqrt(std::max(R(0), R(1) - z * z));
    R phi = R(k) * R(golden_angle()) + jitter * R(2.0 * PI);
    return normalize(V3<R>(r * std::cos(phi), r * std::sin(phi), z));
}

// gi_probes.js:235-251
inline double hysteresis_exponent_for_interval(double dtMs, bool normalize) {
    if (!normalize) return 1;
    const double ref = 1000.0 / 60.0;
    double dt = std::isfinite(dtMs) ? std::max(0.0, dtMs) : ref;
    return std::min(1.0, dt / ref);
}

// gi_probes.js:938-943
inline void compute_grid_resolution(const double size[3], int targetLongAxis, uint32_t out[3]) {
    double longest = std::max(std::max(size[0], size[1]), std::max(size[2], 1e-3));
    double spacing = longest / std::max(1, targetLongAxis);
    for (int a = 0; a < 3; ++a) {
        // THREE.MathUtils.clamp(Math.round(s / spacing) + 1, 2, 32); Math.round = floor(x+0.5)
        double r = std::floor(size[a] / spacing + 0.5) + 1;
        out[a] = (uint32_t)std::min(32.0, std::max(2.0, r));
    }
}

}  // namespace orc
