// sb_trace.cu — the probe trace as a three-stage wavefront (traceKernel,
// gi_probes.js:1977-2214, split where its per-ray work diverges):
//
//   A  k_trace_primary  closest hit per probe ray (traverseClosest) -> raw
//                       16-byte hit record.
//      k_emit           per ray: hit t in double-float, hit frame, and the NEE
//                       pre-tests per candidate light (the reference's
//                       ndl * peak > 0 and range gates); passing candidates
//                       become shadow-ray jobs, one atomic per warp.
//   B  k_trace_shadow   any hit per job (traverseAny); blocked lights are
//                       cleared from the ray's visibility mask.
//   C  k_shade          emissive + unblocked NEE terms (ascending light index,
//                       the reference's summation order) + one-bounce atlas
//                       read, or the SH-9 sky on a miss -> rayData.
//
// A and B are persistent and work-stealing (warps pull 32 items per atomic).
// A issues rays direction-major: a warp holds ray k of 32 neighbouring probes,
// i.e. 32 parallel rays, which keeps the BVH walks of a warp together.
#include "sb_traverse.cuh"

namespace sb {

struct WaveCtx {
    DevScene S;
    DevCascade C;
    DevParams P;
    uint32_t* err;
    unsigned long long* counters;  // [rays, shadowRays, tlasNodes, instances, blasNodes, triTests] or null
    uint32_t* work;                // [0] primary cursor, [1] shadow cursor, [2] job count
    float4* jobs;                  // 2 float4 per job: (origin, maxDist), (dir, ray << 6 | light)
    uint32_t jobCap;
    uint32_t slotBegin, slotCount; // probe slots of this chunk
    uint32_t smemTlas;             // TLAS nodes staged in shared memory (0 = read from global)
    uint32_t order;                // 0 probe-major, 1 direction-major
};

// The TLAS the walk reads (child pairs when `pairs`, else the 32-byte nodes),
// staged in shared memory when it fits.
__device__ __forceinline__ const uint4* stage_tlas(const WaveCtx& W, uint4* sTlas, bool pairs) {
    const DevScene& S = W.S;
    const uint4* src = pairs ? S.tlasPairs : S.tlas;
    if (W.smemTlas >= S.tlasNodeCount && S.tlasNodeCount > 0) {
        const uint32_t n = (pairs ? 4u : 2u) * S.tlasNodeCount;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sTlas[i] = __ldg(src + i);
        __syncthreads();
        return sTlas;
    }
    return src;
}

struct HitFrame {
    float3 ng, hitPos;
    float traceBias;
    bool faceFwd;
};

// Geometric normal through (M^-1)^T, flipped toward the ray, and the biased
// hit position (gi_probes.js:2003-2017).
__device__ __forceinline__ HitFrame hit_frame(const WaveCtx& W, uint32_t tri, uint32_t inst, float3 ro, float3 rd,
                                              float t, int facing) {
    float4 b = __ldg(W.S.tris + 3 * tri + 1), c = __ldg(W.S.tris + 3 * tri + 2);
    float3 nl = normalize3(cross3(xyz(b), xyz(c)));
    float4 r0 = __ldg(W.S.inst + 4 * inst), r1 = __ldg(W.S.inst + 4 * inst + 1), r2 = __ldg(W.S.inst + 4 * inst + 2);
    float3 ngRaw = normalize3(xyz(r0) * nl.x + xyz(r1) * nl.y + xyz(r2) * nl.z);
    HitFrame f;
    f.faceFwd = facing >= 0 ? facing == 1 : dot3(ngRaw, rd) < 0.0f;
    f.ng = ngRaw * (f.faceFwd ? 1.0f : -1.0f);
    f.traceBias = fmaxf(W.C.cellMin * 0.005f * W.P.debugTraceBiasScale, RAY_EPS * W.P.debugRayEpsScale);
    f.hitPos = (ro + rd * t) + f.ng * f.traceBias;
    return f;
}

// Candidate lights of a hit: the C0 cell list in clustered mode
// (gi_probes.js:2109-2127), else every light.
struct LightList {
    const float* list;
    uint32_t count;
};
__device__ __forceinline__ LightList light_list(const WaveCtx& W, float3 hitPos) {
    LightList L{nullptr, W.S.lightCount};
    if (!W.S.clustered) return L;
    const DevCascade& C = W.C;
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
    const float* list = W.S.lights + LIGHT_DATA + cellIndex * 17u;
    uint32_t listCount = (uint32_t)__ldg(list);
    if (outside || listCount > 16u) return L;
    L.list = list;
    L.count = listCount;
    return L;
}
__device__ __forceinline__ uint32_t light_at(const LightList& L, uint32_t i) {
    return L.list ? (uint32_t)__ldg(L.list + 1 + i) : i;
}

struct LightEval {
    float3 wi, lcol, ldir;
    float dist, ndl, lrange, ldecay, lcosAngle, lcosPen;
    bool isDir, isSpot, pass;
};

// The light record and the gates ahead of the shadow query
// (gi_probes.js:2137-2157 / 2066-2084).
__device__ __forceinline__ LightEval light_eval(const WaveCtx& W, uint32_t li, float3 hitPos, float3 ng) {
    const float* L = W.S.lights + li * 17u;
    LightEval e;
    float ltype = __ldg(L);
    e.pass = false;
    if (!(ltype < 2.5f)) return e;
    float3 lpos = mk(__ldg(L + 1), __ldg(L + 2), __ldg(L + 3));
    e.ldir = mk(__ldg(L + 4), __ldg(L + 5), __ldg(L + 6));
    float eclass = __ldg(L + 16);
    bool isIr = fabsf(eclass - 4.0f) < 0.25f;
    float irs = isIr ? W.P.nirGate * W.P.nirGain : 1.0f;
    e.lcol = mk(__ldg(L + 7), __ldg(L + 8), __ldg(L + 9)) * irs;
    e.lrange = __ldg(L + 10);
    e.ldecay = __ldg(L + 11);
    e.lcosAngle = __ldg(L + 12);
    e.lcosPen = __ldg(L + 13);
    e.isDir = ltype < 0.5f;
    e.isSpot = fabsf(ltype - 2.0f) < 0.5f;
    float3 toLight = e.isDir ? e.ldir * -1.0f : lpos - hitPos;
    e.dist = e.isDir ? 1e4f : fmaxf(sqrtf(dot3(toLight, toLight)), 1e-4f);
    e.wi = normalize3(toLight);
    e.ndl = fmaxf(dot3(ng, e.wi), 0.0f);
    float lpeak = fmaxf(fmaxf(e.lcol.x, e.lcol.y), e.lcol.z);
    e.pass = e.ndl * lpeak > 0.0f && (e.isDir || e.lrange <= 0.0f || e.dist < e.lrange);
    return e;
}

// The unshadowed Lambert NEE term (gi_probes.js:2160-2171).
__device__ __forceinline__ float3 light_term(const WaveCtx& W, const LightEval& e, float3 kd) {
    float falloff = 1.0f / fmaxf(powf(e.dist, e.ldecay), 0.01f);
    float rr = e.dist / fmaxf(e.lrange, 1e-4f);
    float rr2 = rr * rr;
    float win = clampf(1.0f - rr2 * rr2, 0.0f, 1.0f);
    float ranged = falloff * (win * win);
    float posAtten = e.lrange > 0.0f ? ranged : falloff;
    float distAtten = e.isDir ? 1.0f : posAtten;
    float angleCos = dot3(e.wi, e.ldir) * -1.0f;
    float spotAtten = clampf((angleCos - e.lcosAngle) / fmaxf(e.lcosPen - e.lcosAngle, 1e-4f), 0.0f, 1.0f);
    float atten = distAtten * (e.isSpot ? spotAtten : 1.0f);
    float3 diffuse = kd * (1.0f / PI_F);
    return mul3(diffuse * e.ndl, e.lcol) * (atten * W.P.debugDirectScale);
}

__device__ __forceinline__ void ray_of(const WaveCtx& W, uint32_t g, bool dirMajor, uint32_t& slot, uint32_t& k) {
    const uint32_t N = W.C.rays;
    uint32_t s;
    if (dirMajor) {
        k = g / W.slotCount;
        s = g - k * W.slotCount;
    } else {
        s = g / N;
        k = g - s * N;
    }
    slot = W.slotBegin + s;
}

// Resident 256-thread blocks per SM the register allocation must allow
// (4 x 256 threads: 64 registers; measured best for both traversal stages).
#ifndef SB_PRIMARY_MIN_BLOCKS
#define SB_PRIMARY_MIN_BLOCKS 4
#endif
#ifndef SB_SHADOW_MIN_BLOCKS
#define SB_SHADOW_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(256, SB_PRIMARY_MIN_BLOCKS) k_trace_primary(WaveCtx W) {
    extern __shared__ uint4 sTlas[];
    const bool pairs = closest_pairs(W.S);
    const uint4* tl = stage_tlas(W, sTlas, pairs);
    if (!*W.S.valid) return;
    const DevCascade& C = W.C;
    const uint32_t N = C.rays, total = W.slotCount * N;
    const uint32_t lane = threadIdx.x & 31u;
    const bool dirMajor = W.order != 0;
    Visits vis = {0, 0, 0, 0};
    uint32_t nRays = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&W.work[0], 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t g = base + lane;
        if (g >= total) continue;
        uint32_t slot, k;
        ray_of(W, g, dirMajor, slot, k);
        const uint32_t probeIndex = (C.probeOffset + slot) % C.probeTotal;
        const float3 ro = probe_world_pos(C, probeIndex);
        const float3 rd = ray_dir(k, N, W.P.frameJitter);
        float bestT, bu, bv;
        int tri, inst;
        trace_closest(W.S, tl, ro, rd, bestT, tri, inst, bu, bv, vis, W.err, pairs);
        ++nRays;
        // raw record (FP32 t, no facing bit): k_emit finishes it
        uint32_t uq = (uint32_t)__float2uint_rn(clampf(bu, 0.f, 1.f) * 65535.0f);
        uint32_t vq = (uint32_t)__float2uint_rn(clampf(bv, 0.f, 1.f) * 65535.0f);
        C.hits[slot * N + k] = tri >= 0 ? make_uint4((uint32_t)tri, (uint32_t)inst, __float_as_uint(bestT),
                                                     uq | (vq << 16))
                                        : make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, __float_as_uint(-1.0f), 0u);
    }
    if (W.counters) {
        atomicAdd(&W.counters[0], (unsigned long long)nRays);
        atomicAdd(&W.counters[2], (unsigned long long)vis.tlas);
        atomicAdd(&W.counters[3], (unsigned long long)vis.inst);
        atomicAdd(&W.counters[4], (unsigned long long)vis.blas);
        atomicAdd(&W.counters[5], (unsigned long long)vis.tri);
    }
}

// Stage A2, one thread per probe ray in the issue order of A: the hit
// parameter re-evaluated in double-float, the hit frame, and the NEE gates of
// every candidate light. Each lane runs the gates with no warp sync; one warp
// scan and one atomicAdd then reserve the warp's shadow-ray jobs, and each
// ray's passing candidates (gates evaluated again: the same pure function) are
// written together in list order, so a shadow warp mostly holds rays that share
// an origin.
__global__ void __launch_bounds__(128) k_emit(WaveCtx W) {
    if (!*W.S.valid) return;
    const DevCascade& C = W.C;
    const uint32_t N = C.rays, total = W.slotCount * N;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t rayIdx = 0;
    int tri = -1;
    HitFrame fr;
    fr.hitPos = mk(0.f, 0.f, 0.f);
    fr.ng = mk(0.f, 0.f, 1.f);
    fr.faceFwd = true;
    fr.traceBias = 0.f;
    uint4 h = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u);
    if (g < total) {
        uint32_t slot, k;
        ray_of(W, g, W.order != 0, slot, k);
        rayIdx = slot * N + k;
        h = C.hits[rayIdx];
        if (h.x != 0xFFFFFFFFu) {
            tri = (int)h.x;
            const uint32_t inst = h.y;
            const float3 ro = probe_world_pos(C, (C.probeOffset + slot) % C.probeTotal);
            const float3 rd = ray_dir(k, N, W.P.frameJitter);
            const float t = refine_t(W.S, (uint32_t)tri, inst, ro, rd);
            fr = hit_frame(W, (uint32_t)tri, inst, ro, rd, t, -1);
            h.y = inst | (fr.faceFwd ? 0x80000000u : 0u);
            h.z = __float_as_uint(t);
        }
    }
    LightList L{nullptr, 0u};
    if (tri >= 0) L = light_list(W, fr.hitPos);
    unsigned long long pass = 0ull;
    for (uint32_t i = 0; i < L.count; ++i)
        if (light_eval(W, light_at(L, i), fr.hitPos, fr.ng).pass) pass |= 1ull << i;
    const uint32_t mine = (uint32_t)__popcll(pass);
    uint32_t incl = mine;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += v;
    }
    const uint32_t warpJobs = __shfl_sync(0xFFFFFFFFu, incl, 31);
    uint32_t jb = 0;
    if (warpJobs) {
        if (lane == 0) jb = atomicAdd(&W.work[2], warpJobs);
        jb = __shfl_sync(0xFFFFFFFFu, jb, 0);
    }
    uint32_t j = jb + incl - mine, tested0 = 0u, tested1 = 0u, nJobs = 0;
    while (pass) {
        const uint32_t i = (uint32_t)(__ffsll((long long)pass) - 1);
        pass &= pass - 1ull;
        const uint32_t li = light_at(L, i);
        const LightEval e = light_eval(W, li, fr.hitPos, fr.ng);
        if (j < W.jobCap) {
            W.jobs[2 * j] = make_float4(fr.hitPos.x, fr.hitPos.y, fr.hitPos.z, e.dist - fr.traceBias);
            W.jobs[2 * j + 1] = make_float4(e.wi.x, e.wi.y, e.wi.z, __uint_as_float((rayIdx << 6) | li));
            if (li < 32) tested0 |= 1u << li;
            else tested1 |= 1u << (li - 32);
            ++nJobs;
        } else {
            latch(W.err, ERR_CAPACITY);
        }
        ++j;
    }
    if (g < total) {
        if (tri >= 0) C.hits[rayIdx] = h;
        C.vis[rayIdx] = make_uint4(tested0, tested1, tested0, tested1);
    }
    if (W.counters) {
        const uint32_t warpDone = __reduce_add_sync(0xFFFFFFFFu, nJobs);
        if (lane == 0 && warpDone) atomicAdd(&W.counters[1], (unsigned long long)warpDone);
    }
}

__global__ void __launch_bounds__(256, SB_SHADOW_MIN_BLOCKS) k_trace_shadow(WaveCtx W) {
    extern __shared__ uint4 sTlas[];
    const bool pairs = any_pairs(W.S);
    const uint4* tl = stage_tlas(W, sTlas, pairs);
    if (!*W.S.valid) return;
    const uint32_t total = min(*(volatile uint32_t*)&W.work[2], W.jobCap);
    const uint32_t lane = threadIdx.x & 31u;
    Visits vis = {0, 0, 0, 0};
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&W.work[1], 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        uint32_t j = base + lane;
        if (j >= total) continue;
        float4 a = W.jobs[2 * j], b = W.jobs[2 * j + 1];
        if (trace_any(W.S, tl, xyz(a), xyz(b), a.w, vis, W.err, pairs)) {
            uint32_t packed = __float_as_uint(b.w);
            uint32_t ray = packed >> 6, li = packed & 63u;
            uint4* v = W.C.vis + ray;
            if (li < 32) atomicAnd(&v->z, ~(1u << li));
            else atomicAnd(&v->w, ~(1u << (li - 32)));
        }
    }
    if (W.counters) {
        atomicAdd(&W.counters[6], (unsigned long long)vis.tlas);
        atomicAdd(&W.counters[7], (unsigned long long)vis.inst);
        atomicAdd(&W.counters[8], (unsigned long long)vis.blas);
        atomicAdd(&W.counters[9], (unsigned long long)vis.tri);
    }
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

__global__ void __launch_bounds__(128) k_shade(WaveCtx W) {
    if (!*W.S.valid) return;
    const DevCascade& C = W.C;
    const uint32_t N = C.rays;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= W.slotCount * N) return;
    uint32_t slot, k;
    ray_of(W, g, false, slot, k);
    const uint32_t rayIdx = slot * N + k;
    uint32_t probeIndex = (C.probeOffset + slot) % C.probeTotal;
    float3 ro = probe_world_pos(C, probeIndex);
    float3 rd = ray_dir(k, N, W.P.frameJitter);
    uint4 h = C.hits[rayIdx];
    float3 outRgb;
    float hitT = -1.0f;
    if (h.x != 0xFFFFFFFFu) {
        uint32_t tri = h.x, inst = h.y & 0x7FFFFFFFu;
        float t = __uint_as_float(h.z);
        hitT = t;
        HitFrame fr = hit_frame(W, tri, inst, ro, rd, t, (int)(h.y >> 31));
        uint32_t m = __ldg(W.S.triMaterial + tri);
        const float* M = W.S.materials + (size_t)m * 28u;
        float3 baseColor = mk(__ldg(M), __ldg(M + 1), __ldg(M + 2));
        float3 emissive = mk(__ldg(M + 7), __ldg(M + 8), __ldg(M + 9));
        float3 radiance = emissive * W.P.debugEmissiveScale;
        float metal = __ldg(M + 4), transm = __ldg(M + 5);
        float3 kdr = baseColor * W.P.debugAlbedoScale * (1.0f - metal) * (1.0f - transm);
        float3 kd = mk(clampf(kdr.x, 0.f, 0.95f), clampf(kdr.y, 0.f, 0.95f), clampf(kdr.z, 0.f, 0.95f));
        uint4 v = C.vis[rayIdx];
        unsigned long long ok = (unsigned long long)v.z | ((unsigned long long)v.w << 32);
        while (ok) {
            uint32_t li = (uint32_t)(__ffsll((long long)ok) - 1);
            ok &= ok - 1ull;
            LightEval e = light_eval(W, li, fr.hitPos, fr.ng);
            radiance = radiance + light_term(W, e, kd);
        }
        float3 bounce = mul3(sample_atlas(C, fr.hitPos, fr.ng), kd) * (1.0f / PI_F);
        float bl = luma3(bounce);
        float roll = W.P.radianceClamp / fmaxf(fmaxf(W.P.radianceClamp, bl), 1e-6f);
        outRgb = radiance + bounce * roll * W.P.debugBounceScale;
    } else {
        outRgb = sky_sh(W.P, rd);
    }
    C.rayData[rayIdx] = make_float4(outRgb.x, outRgb.y, outRgb.z, hitT);
}

static int persistent_grid(const void* kernel, int block, size_t smem, const TraceTuning& tune, uint32_t items) {
    int perSm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, block, smem);
    if (perSm < 1) perSm = 1;
    int grid = tune.numSms * perSm;
    uint32_t needed = (items + block - 1) / block;
    if ((uint32_t)grid > needed) grid = (int)needed;
    return grid < 1 ? 1 : grid;
}

cudaError_t launch_trace(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t* err,
                         unsigned long long* counters, uint32_t* work, const TraceTuning& tune, cudaStream_t st,
                         float4* jobs, uint32_t jobCap, uint32_t slotBegin, uint32_t slotCount,
                         cudaEvent_t afterPrimary, cudaEvent_t afterShadow) {
    if (slotCount == 0) return cudaSuccess;
    WaveCtx W;
    W.S = S;
    W.C = C;
    W.P = P;
    W.err = err;
    W.counters = counters;
    W.work = work;
    W.jobs = jobs;
    W.jobCap = jobCap;
    W.slotBegin = slotBegin;
    W.slotCount = slotCount;
    W.order = tune.sortKey == 0 ? 1u : 0u;  // default direction-major; sortKey 1 = probe-major
    // the scene-BVH walk reads no TLAS
    uint32_t smemNodes = !S.flatOn && S.tlasNodeCount <= tune.smemTlasNodes ? S.tlasNodeCount : 0u;
    W.smemTlas = smemNodes;
    size_t smem = (size_t)smemNodes * 64u;  // room for the child-pair TLAS (the 32-byte nodes need half)
    if (smem > 48u * 1024u) {
        cudaFuncSetAttribute(k_trace_primary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_trace_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    cudaError_t e = cudaMemsetAsync(work, 0, 3 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t rays = slotCount * C.rays;
    int block = (int)tune.block;
    k_trace_primary<<<persistent_grid((const void*)k_trace_primary, block, smem, tune, rays), block, smem, st>>>(W);
    note_launch();
    k_emit<<<(rays + 127) / 128, 128, 0, st>>>(W);
    note_launch();
    if (afterPrimary) cudaEventRecord(afterPrimary, st);
    // shadow jobs: at most lightCount per ray (the queue is sized for it)
    k_trace_shadow<<<persistent_grid((const void*)k_trace_shadow, block, smem, tune, rays * 4u), block, smem, st>>>(W);
    note_launch();
    if (afterShadow) cudaEventRecord(afterShadow, st);
    k_shade<<<(rays + 127) / 128, 128, 0, st>>>(W);
    note_launch();
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
    const bool pairs = closest_pairs(S);
    trace_closest(S, pairs ? S.tlasPairs : S.tlas, o, d, t, tri, inst, bu, bv, vis, err, pairs);
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
    const bool pairs = any_pairs(S);
    out[i] = trace_any(S, pairs ? S.tlasPairs : S.tlas, mk(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]),
                       mk(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]), maxDist[i], vis, err, pairs)
                 ? 1
                 : 0;
}

cudaError_t launch_raycast(const DevScene& S, const float* ro, const float* rd, uint32_t n, float* tOut,
                           int32_t* triOut, int32_t* instOut, uint32_t* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_raycast<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, n, tOut, triOut, instOut, err);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_occluded(const DevScene& S, const float* ro, const float* rd, const float* maxDist, uint32_t n,
                            uint8_t* out, uint32_t* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_occluded<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, maxDist, n, out, err);
    note_launch();
    return cudaGetLastError();
}

}  // namespace sb
