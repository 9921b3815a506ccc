// sb_cascade.cu — placement of the fine cascade C1 (fitFineBox,
// gi_probes.js:2963-3030): a 16^3 density histogram of the pooled
// triangles' centroids over the coarse box, the bins of at least 0.4 x the
// peak united into a box, padded by one bin, its extent clamped per axis to
// [0.25, 0.60] of the coarse box and slid back inside it.
//
// The histogram runs on the GPU over the pool already resident there (one
// thread per triangle, one atomic per triangle into 4,096 bins). The reference
// computes the bin index in JS doubles (centroid, offset, scale, ToInt32), and
// a centroid on a bin edge lands in the bin the double arithmetic picks, so the
// kernel evaluates those few operations in FP64 with each one rounded as JS
// rounds it; the 4,096-bin reduction and the box arithmetic after it run on
// the host in doubles, in the reference's order.
#include <cmath>

#include "sb_kernels.cuh"

namespace sb {

namespace {

constexpr int kG = 16;

// ECMAScript ToInt32 of a double (the `| 0` of gi_probes.js:2981-2983).
__device__ __forceinline__ int32_t js_to_int32(double x) {
    if (!isfinite(x)) return 0;
    double t = trunc(x);
    double m = fmod(t, 4294967296.0);
    if (m < 0.0) m += 4294967296.0;
    if (m >= 2147483648.0) m -= 4294967296.0;
    return (int32_t)m;
}

__global__ void k_fine_hist(const uint32_t* triIndex, const float* vertexData, uint32_t T, double3 mn, double3 inv,
                            uint32_t* hist) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for (int k = 0; k < 3; ++k) {
        const float* v = vertexData + (size_t)triIndex[3 * (size_t)t + k] * 8u;
        cx = __dadd_rn(cx, (double)v[0]);
        cy = __dadd_rn(cy, (double)v[1]);
        cz = __dadd_rn(cz, (double)v[2]);
    }
    cx = __ddiv_rn(cx, 3.0);
    cy = __ddiv_rn(cy, 3.0);
    cz = __ddiv_rn(cz, 3.0);
    const int gx = min(max(js_to_int32(__dmul_rn(__dsub_rn(cx, mn.x), inv.x)), 0), kG - 1);
    const int gy = min(max(js_to_int32(__dmul_rn(__dsub_rn(cy, mn.y), inv.y)), 0), kG - 1);
    const int gz = min(max(js_to_int32(__dmul_rn(__dsub_rn(cz, mn.z), inv.z)), 0), kG - 1);
    atomicAdd(hist + (gz * kG + gy) * kG + gx, 1u);
}

}  // namespace

cudaError_t launch_fine_hist(const SceneBuffers& B, const double mn[3], const double inv[3], uint32_t* hist,
                             cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(hist, 0, kG * kG * kG * sizeof(uint32_t), st);
    if (e != cudaSuccess || B.triCount == 0) return e;
    k_fine_hist<<<(B.triCount + 255) / 256, 256, 0, st>>>(B.triIndex, B.vertexData, B.triCount,
                                                           make_double3(mn[0], mn[1], mn[2]),
                                                           make_double3(inv[0], inv[1], inv[2]), hist);
    note_launch();
    return cudaGetLastError();
}

// The host half of fitFineBox over the histogram (gi_probes.js:2988-3029).
bool fine_box_from_hist(const uint32_t* hist, const double mn[3], const double size[3], double outMin[3],
                        double outSize[3]) {
    const int G = kG;
    uint32_t peak = 0;
    for (int i = 0; i < G * G * G; ++i)
        if (hist[i] > peak) peak = hist[i];
    if (peak == 0) return false;
    const double thr = (double)peak * 0.4;  // C1_HIST_THRESHOLD
    int bx0 = G, by0 = G, bz0 = G, bx1 = -1, by1 = -1, bz1 = -1, count = 0;
    for (int z = 0; z < G; ++z)
        for (int y = 0; y < G; ++y)
            for (int x = 0; x < G; ++x)
                if ((double)hist[(z * G + y) * G + x] >= thr) {
                    if (x < bx0) bx0 = x;
                    if (x > bx1) bx1 = x;
                    if (y < by0) by0 = y;
                    if (y > by1) by1 = y;
                    if (z < bz0) bz0 = z;
                    if (z > bz1) bz1 = z;
                    ++count;
                }
    if (count == 0 || bx1 < 0) return false;
    if (bx0 == 0 && by0 == 0 && bz0 == 0 && bx1 == G - 1 && by1 == G - 1 && bz1 == G - 1) return false;
    const double cell[3] = {size[0] / G, size[1] / G, size[2] / G};
    double fmin[3] = {mn[0] + bx0 * cell[0], mn[1] + by0 * cell[1], mn[2] + bz0 * cell[2]};
    double fmax[3] = {mn[0] + (bx1 + 1) * cell[0], mn[1] + (by1 + 1) * cell[1], mn[2] + (bz1 + 1) * cell[2]};
    const double pad = std::fmin(std::fmin(cell[0], cell[1]), cell[2]);
    for (int a = 0; a < 3; ++a) {
        fmin[a] -= pad;
        fmax[a] += pad;
    }
    double fsize[3] = {fmax[0] - fmin[0], fmax[1] - fmin[1], fmax[2] - fmin[2]};
    const double box0max[3] = {mn[0] + size[0], mn[1] + size[1], mn[2] + size[2]};
    for (int a = 0; a < 3; ++a) {
        const double lo = 0.25 * size[a];  // C1_MIN_AXIS_FRAC
        const double hi = 0.60 * size[a];  // C1_MAX_AXIS_FRAC
        const double s = std::fmax(lo, std::fmin(hi, fsize[a]));  // THREE.MathUtils.clamp
        const double center = (fmin[a] + fmax[a]) * 0.5;
        double lo2 = center - s * 0.5;
        double hi2 = center + s * 0.5;
        if (lo2 < mn[a]) {
            hi2 += (mn[a] - lo2);
            lo2 = mn[a];
        }
        if (hi2 > box0max[a]) {
            lo2 -= (hi2 - box0max[a]);
            hi2 = box0max[a];
        }
        lo2 = std::fmax(lo2, mn[a]);
        hi2 = std::fmin(hi2, box0max[a]);
        fmin[a] = lo2;
        fsize[a] = std::fmax(1e-4, hi2 - lo2);
    }
    for (int a = 0; a < 3; ++a) {
        outMin[a] = fmin[a];
        outSize[a] = fsize[a];
    }
    return true;
}

}  // namespace sb
