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
#include "sb_wave.cuh"

namespace sb {

// Resident 256-thread blocks per SM the register allocation must allow
// (4 x 256 threads: 64 registers; measured best for both traversal stages).
#ifndef SB_PRIMARY_MIN_BLOCKS
#define SB_PRIMARY_MIN_BLOCKS 4
#endif
#ifndef SB_SHADOW_MIN_BLOCKS
#define SB_SHADOW_MIN_BLOCKS 4
#endif
// Group-stack entries per thread held in shared memory by the closest-hit
// stage's 8-wide walk (8 bytes each, one [entry][thread] array per CTA) when
// the tree's depth fits; 0, or a deeper tree: the stack in local memory.
#ifndef SB_SMEM_STACK
#define SB_SMEM_STACK 16
#endif

// ---------------------------------------------------------------- bodies
// Each stage's per-item work is a device function over `const WaveCtx&`; the
// per-solve kernels pass their parameter, the batched kernels an item of the
// __grid_constant__ BatchArgs (indexed in the parameter space, warp-uniform).

__device__ __forceinline__ void add_visits(unsigned long long* c, int at, uint32_t rays, const Visits& v) {
    if (!c) return;
    if (rays) atomicAdd(&c[0], (unsigned long long)rays);
    atomicAdd(&c[at], (unsigned long long)v.tlas);
    atomicAdd(&c[at + 1], (unsigned long long)v.inst);
    atomicAdd(&c[at + 2], (unsigned long long)v.blas);
    atomicAdd(&c[at + 3], (unsigned long long)v.tri);
}

// The raw record of a closest hit (FP32 t, no facing bit): k_emit finishes it.
__device__ __forceinline__ void write_hit(const DevCascade& C, uint32_t slot, uint32_t k, int tri, int inst, float t,
                                          float bu, float bv) {
    const uint32_t uq = (uint32_t)__float2uint_rn(clampf(bu, 0.f, 1.f) * 65535.0f);
    const uint32_t vq = (uint32_t)__float2uint_rn(clampf(bv, 0.f, 1.f) * 65535.0f);
    C.hits[slot * C.rays + k] = tri >= 0 ? make_uint4((uint32_t)tri, (uint32_t)inst, __float_as_uint(t), uq | (vq << 16))
                                         : make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, __float_as_uint(-1.0f), 0u);
}

// Stage A: the closest hit of one probe ray (item-local issue index g).
__device__ __forceinline__ void primary_ray(const WaveCtx& W, const uint4* tl, bool pairs, uint32_t g, Visits& vis,
                                            const uint4* sWide = nullptr, uint32_t nWide = 0) {
    const DevCascade& C = W.C;
    uint32_t slot, k;
    ray_of(W, g, W.order != 0, slot, k);
    const uint32_t probeIndex = (C.probeOffset + slot) % C.probeTotal;
    const float3 ro = probe_world_pos(C, probeIndex);
    const float3 rd = ray_dir(k, C.rays, W.P.frameJitter);
    float bestT, bu, bv;
    int tri, inst;
    trace_closest(W.S, tl, ro, rd, bestT, tri, inst, bu, bv, vis, W.err, pairs, sWide, nWide);
    write_hit(C, slot, k, tri, inst, bestT, bu, bv);
}

// Stage A on the 8-wide tree with per-lane refill, for a whole persistent warp
// (all 32 lanes call it): each lane walks its own ray in rounds (wide_step),
// and a lane whose walk has ended takes the next ray of the issue order before
// the next round, so the lanes keep working instead of waiting for the slowest
// ray of a fixed 32-ray batch. One atomicAdd per round fetches rays for all
// the warp's idle lanes. Returns the rays traced.
//
// sStack: this thread's column of the walk stack in shared memory (W.sstk
// entries), or null for the stack in local memory.
__device__ __forceinline__ uint32_t primary_refill(const WaveCtx& W, uint32_t total, Visits& vis, const uint4* sWide,
                                                   uint32_t nWide, uint2* sStack = nullptr) {
    const DevCascade& C = W.C;
    const uint32_t lane = threadIdx.x & 31u;
    WideWalk w;
    uint32_t slot = 0, k = 0, nRays = 0;
    float bestT = T_MAX, bu = 0.0f, bv = 0.0f;
    int tri = -1, inst = -1;
    bool has = false, more = true;
    for (;;) {
        if (more) {
            const uint32_t need = __ballot_sync(0xFFFFFFFFu, !has);
            if (need) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&W.work[0], (uint32_t)__popc(need));
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= total) more = false;
                const uint32_t g = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
                if (!has && g < total) {
                    ray_of(W, g, W.order != 0, slot, k);
                    const float3 ro = probe_world_pos(C, (C.probeOffset + slot) % C.probeTotal);
                    const float3 rd = ray_dir(k, C.rays, W.P.frameJitter);
                    bestT = T_MAX;
                    tri = inst = -1;
                    bu = bv = 0.0f;
                    wide_begin<false>(W.S, w, ro, rd, bestT, tri, inst, bu, bv, vis, W.err);
                    has = true;
                }
            }
        }
        if (!__any_sync(0xFFFFFFFFu, has)) {
            if (!more) break;
            continue;
        }
        if (has && wide_step<false>(W.S, w, bestT, tri, inst, bu, bv, vis, W.err, sWide, nWide, sStack,
                                    (int)W.sstk)) {
            wide_end<false>(W.S, w, bestT, tri, inst, bu, bv, vis, W.err);
            write_hit(C, slot, k, tri, inst, bestT, bu, bv);
            ++nRays;
            has = false;
        }
    }
    return nRays;
}

// Stage A2, warp-collective (all 32 lanes call it; `active` lanes hold ray g):
// the hit parameter re-evaluated in double-float, the hit frame, and the NEE
// gates of every candidate light. Each lane runs the gates with no warp sync;
// one warp scan and one atomicAdd then reserve the warp's shadow-ray jobs, and
// each ray's passing candidates (gates evaluated again: the same pure
// function) are written together in list order, so a shadow warp mostly holds
// rays that share an origin. Jobs carry tagBase + the ray's record index.
__device__ __forceinline__ uint32_t emit_ray(const WaveCtx& W, bool active, uint32_t g, uint32_t tagBase) {
    const DevCascade& C = W.C;
    const uint32_t N = C.rays;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t rayIdx = 0;
    int tri = -1;
    HitFrame fr;
    fr.hitPos = mk(0.f, 0.f, 0.f);
    fr.ng = mk(0.f, 0.f, 1.f);
    fr.faceFwd = true;
    fr.traceBias = 0.f;
    uint4 h = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u);
    if (active) {
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
        if (light_gate(W, light_at(L, i), fr.hitPos, fr.ng)) pass |= 1ull << i;
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
    const uint32_t tag = (tagBase + rayIdx) << 6;
    while (pass) {
        const uint32_t i = (uint32_t)(__ffsll((long long)pass) - 1);
        pass &= pass - 1ull;
        const uint32_t li = light_at(L, i);
        if (j < W.jobCap) {
            float3 wi;
            float dist;
            light_ray(W, li, fr.hitPos, wi, dist);
            W.jobs[2 * j] = make_float4(fr.hitPos.x, fr.hitPos.y, fr.hitPos.z, dist - fr.traceBias);
            W.jobs[2 * j + 1] = make_float4(wi.x, wi.y, wi.z, __uint_as_float(tag | li));
            if (li < 32) tested0 |= 1u << li;
            else tested1 |= 1u << (li - 32);
            ++nJobs;
        } else {
            latch(W.err, ERR_CAPACITY);
        }
        ++j;
    }
    if (active) {
        if (tri >= 0) C.hits[rayIdx] = h;
        C.vis[rayIdx] = make_uint4(tested0, tested1, tested0, tested1);
    }
    return nJobs;
}

// Stage B: one shadow job; a blocked light is cleared from the ray's mask.
__device__ __forceinline__ void shadow_job(const WaveCtx& W, const uint4* tl, bool pairs, float4 a, float4 b,
                                           uint32_t rayIdx, Visits& vis) {
    if (trace_any(W.S, tl, xyz(a), xyz(b), a.w, vis, W.err, pairs)) {
        const uint32_t li = __float_as_uint(b.w) & 63u;
        uint4* v = W.C.vis + rayIdx;
        if (li < 32) atomicAnd(&v->z, ~(1u << li));
        else atomicAnd(&v->w, ~(1u << (li - 32)));
    }
}

// Stage C: emissive + unblocked NEE terms + bounce, or the sky, of one ray
// (item-local probe-major index g).
__device__ __forceinline__ void shade_ray(const WaveCtx& W, uint32_t g) {
    const DevCascade& C = W.C;
    const uint32_t N = C.rays;
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
        if (C.reflect) {
            // with the reflection lobes on, a hit on a surface with no diffuse energy
            // and no emission is stored as -(t + 2): the blend keeps its depth, the
            // lobes ignore it (gi_probes.js:2055-2062)
            const float diffuseEnergy = (1.0f - metal) * (1.0f - transm);
            const float emissivePeak = fmaxf(fmaxf(emissive.x, emissive.y), emissive.z);
            if (!(diffuseEnergy > 0.02f || emissivePeak > 1e-6f)) hitT = -(t + ROUGH_UNSHADED_T_BIAS);
        }
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

// ---------------------------------------------------------------- per solve

__global__ void __launch_bounds__(256, SB_PRIMARY_MIN_BLOCKS) k_trace_primary(WaveCtx W) {
    extern __shared__ uint4 sTlas[];
    const bool pairs = closest_pairs(W.S);
    const uint4* tl = stage_tlas(W, sTlas, pairs);
    // the scene BVH's top 8-wide nodes (the TLAS is not read on that walk:
    // the buffer is free), staged once per CTA
    const uint32_t nWide = W.S.wideNodes ? W.smemWide : 0u;
    if (nWide) {
        for (uint32_t i = threadIdx.x; i < 5u * nWide; i += blockDim.x) sTlas[i] = __ldg(W.S.wideNodes + i);
        __syncthreads();
    }
    if (!*W.S.valid) return;
    const uint32_t total = W.slotCount * W.C.rays;
    const uint32_t lane = threadIdx.x & 31u;
    Visits vis = {0, 0, 0, 0};
    uint32_t nRays = 0;
    if (SB_PRIMARY_REFILL && W.S.wideNodes) {
        // the walk stack after the staged nodes, one column per thread
        uint2* sStack = W.sstk ? reinterpret_cast<uint2*>(sTlas + 5u * nWide) + threadIdx.x : nullptr;
        nRays = primary_refill(W, total, vis, sTlas, nWide, sStack);
        add_visits(W.counters, 2, nRays, vis);
        return;
    }
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&W.work[0], 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        // the batch at this issue position: costliest first when an order is given
        // (a permutation of the (total + 31) / 32 batches; clamped all the same)
        const uint32_t batch =
            W.C.batchOrder ? min(__ldg(W.C.batchOrder + (base >> 5)), (total - 1u) >> 5) : base >> 5;
        const uint32_t g = batch * 32u + lane;
        const long long t0 = W.C.batchCost ? clock64() : 0;
        if (g < total) {
            primary_ray(W, tl, pairs, g, vis, sTlas, nWide);
            ++nRays;
        }
        if (W.C.batchCost) {
            __syncwarp();
            if (lane == 0) W.C.batchCost[batch] = (uint32_t)min(clock64() - t0, 0xFFFFFFFFll);
        }
    }
    add_visits(W.counters, 2, nRays, vis);
}

// The closest-hit batch order for the next full solve, by one CTA (all its
// threads call it; blockDim a multiple of 32): batches by descending recorded
// cycles, a counting sort over 128 log-spaced bins (4 per octave), so the
// persistent kernel starts the long batches first and its last warps hold
// short ones. Order within a bin is arbitrary; results do not depend on it.
__device__ __forceinline__ uint32_t cost_bin(uint32_t c) {
    if (c < 4u) return 0u;
    const uint32_t msb = 31u - __clz(c);
    return min(127u, msb * 4u + ((c >> (msb - 2u)) & 3u));
}
__device__ void order_batches(const uint32_t* cost, uint32_t* order, uint32_t n, uint32_t* at /* shared, 128 */) {
    for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) at[i] = 0u;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&at[cost_bin(__ldcg(cost + i))], 1u);
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan from the costliest bin down: 4 bins per lane
        const uint32_t l = threadIdx.x;
        uint32_t v[4], sum = 0;
        for (uint32_t j = 0; j < 4; ++j) {
            v[j] = at[127u - (4u * l + j)];
            sum += v[j];
        }
        uint32_t incl = sum;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (l >= d) incl += u;
        }
        uint32_t run = incl - sum;
        for (uint32_t j = 0; j < 4; ++j) {
            at[127u - (4u * l + j)] = run;
            run += v[j];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) order[atomicAdd(&at[cost_bin(__ldcg(cost + i))], 1u)] = i;
}

__global__ void __launch_bounds__(128) k_emit(WaveCtx W) {
    if (!*W.S.valid) return;
    const uint32_t total = W.slotCount * W.C.rays;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nJobs = emit_ray(W, g < total, g, 0u);
    if (W.counters) {
        const uint32_t warpDone = __reduce_add_sync(0xFFFFFFFFu, nJobs);
        if ((threadIdx.x & 31u) == 0 && warpDone) atomicAdd(&W.counters[1], (unsigned long long)warpDone);
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
        const float4 a = W.jobs[2 * j], b = W.jobs[2 * j + 1];
        shadow_job(W, tl, pairs, a, b, __float_as_uint(b.w) >> 6, vis);
    }
    add_visits(W.counters, 6, 0u, vis);
    if (W.C.batchOrderOut) {
        // the queue is drained: the first CTA whose warps are all done orders the
        // closest-hit batches for the next solve while the others finish their jobs
        __shared__ uint32_t at[128];
        __shared__ uint32_t first;
        __syncthreads();
        if (threadIdx.x == 0) first = atomicAdd(&W.work[3], 1u) == 0u ? 1u : 0u;
        __syncthreads();
        if (first) order_batches(W.C.batchCost, W.C.batchOrderOut, (W.slotCount * W.C.rays + 31u) / 32u, at);
    }
}

__global__ void __launch_bounds__(128) k_shade(WaveCtx W) {
    if (!*W.S.valid) return;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= W.slotCount * W.C.rays) return;
    shade_ray(W, g);
}

// Stage C alone over probe slots [0, slotCount) from the records already in
// C.hits / C.vis (the adjoint re-evaluates shading this way).
cudaError_t launch_shade(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t slotCount,
                         cudaStream_t st) {
    if (slotCount == 0) return cudaSuccess;
    WaveCtx W{};
    W.S = S;
    W.C = C;
    W.P = P;
    W.slotBegin = 0;
    W.slotCount = slotCount;
    const uint32_t rays = slotCount * C.rays;
    k_shade<<<(rays + 127) / 128, 128, 0, st>>>(W);
    note_launch();
    return cudaGetLastError();
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
                         cudaEvent_t afterPrimary, cudaEvent_t afterShadow, cudaEvent_t afterClosest) {
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
    W.order = tune.sortKey == 1 ? 0u : 1u;  // direction-major (sortKey 0, and 2 over probe tiles); 1 = probe-major
    // the scene-BVH walk reads no TLAS
    uint32_t smemNodes = !S.flatOn && S.tlasNodeCount <= tune.smemTlasNodes ? S.tlasNodeCount : 0u;
    W.smemTlas = smemNodes;
    // the 8-wide walk's top nodes, staged by the closest-hit stage only
    uint32_t wideNodes = S.wideNodes ? (tune.smemWideNodes < S.wideNodeCount ? tune.smemWideNodes : S.wideNodeCount) : 0u;
    if (wideNodes > 512u) wideNodes = 512u;
    W.smemWide = wideNodes;
    size_t smem = (size_t)smemNodes * 64u;  // room for the child-pair TLAS (the 32-byte nodes need half)
    size_t smemPrimary = smem > (size_t)wideNodes * 80u ? smem : (size_t)wideNodes * 80u;
    // the walk stack in shared memory when the 8-wide tree's depth fits it (the
    // stack holds at most one group per level below the root)
    W.sstk = (SB_PRIMARY_REFILL && S.wideNodes && S.wideDepth + 1u <= (uint32_t)SB_SMEM_STACK) ? SB_SMEM_STACK : 0u;
    smemPrimary += (size_t)W.sstk * (size_t)tune.block * 8u;
    if (smemPrimary > 48u * 1024u)
        cudaFuncSetAttribute(k_trace_primary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemPrimary);
    if (smem > 48u * 1024u)
        cudaFuncSetAttribute(k_trace_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // ray, job-read and job-write cursors, and the batch-order claim
    cudaError_t e = cudaMemsetAsync(work, 0, 4 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t rays = slotCount * C.rays;
    int block = (int)tune.block;
    k_trace_primary<<<persistent_grid((const void*)k_trace_primary, block, smemPrimary, tune, rays), block, smemPrimary,
                      st>>>(W);
    note_launch();
    if (afterClosest) cudaEventRecord(afterClosest, st);
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

// ---------------------------------------------------------------- batched
// The same four stages over every item of a BatchArgs: one launch per stage
// for all scenes and cascades, one shared ray index space and job queue.

__global__ void __launch_bounds__(256, SB_PRIMARY_MIN_BLOCKS) k_trace_primary_batch(const __grid_constant__ BatchArgs B) {
    const uint32_t lane = threadIdx.x & 31u;
    Visits vis = {0, 0, 0, 0};
    uint32_t nRays = 0;
    if (!SB_PRIMARY_REFILL) {
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&B.work[0], 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= B.totalRays) break;
            const BatchItem& I = B.it[batch_item(B, base)];
            const uint32_t g = base + lane - I.rayBase;
            if (g >= I.rays || !*I.W.S.valid) continue;
            const bool pairs = closest_pairs(I.W.S);
            primary_ray(I.W, pairs ? I.W.S.tlasPairs : I.W.S.tlas, pairs, g, vis);
            ++nRays;
        }
        add_visits(B.counters, 2, nRays, vis);
        return;
    }
    // Per-lane refill within one item at a time (the item index stays
    // warp-uniform, so the parameter-space reads of its context stay uniform):
    // the warp takes 32-ray chunks and hands their rays to idle lanes; a chunk
    // of another item waits until every lane is idle. Items without an 8-wide
    // tree run their chunks as 32-ray batches (primary_ray).
    const uint32_t NONE = 0xFFFFFFFFu;
    uint32_t item = NONE, cur = 0, curEnd = 0, pend = NONE;  // warp-uniform
    bool more = true;
    WideWalk w;
    uint32_t slot = 0, k = 0;
    float bestT = T_MAX, bu = 0.0f, bv = 0.0f;
    int tri = -1, inst = -1;
    bool has = false;
    for (;;) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !has);
        if (cur == curEnd) {
            if (pend == NONE && more) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&B.work[0], 32u);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= B.totalRays) more = false;
                else pend = base;
            }
            if (pend != NONE) {
                const uint32_t pi = batch_item(B, pend);
                if (pi == item || need == 0xFFFFFFFFu) {
                    const BatchItem& P = B.it[pi];
                    item = pi;
                    cur = pend;
                    curEnd = min(pend + 32u, P.rayBase + P.rays);  // item ranges are 32-aligned
                    if (cur > curEnd || !*P.W.S.valid) cur = curEnd;
                    pend = NONE;
                }
            }
        }
        if (cur < curEnd) {
            const BatchItem& I = B.it[item];
            if (!I.W.S.wideNodes) {
                if (need == 0xFFFFFFFFu) {  // a 32-ray batch, as without refill
                    const uint32_t g = cur + lane - I.rayBase;
                    if (cur + lane < curEnd) {
                        const bool pairs = closest_pairs(I.W.S);
                        primary_ray(I.W, pairs ? I.W.S.tlasPairs : I.W.S.tlas, pairs, g, vis);
                        ++nRays;
                    }
                    cur = curEnd;
                }
            } else if (need) {
                const uint32_t rank = (uint32_t)__popc(need & ((1u << lane) - 1u));
                const uint32_t n = min((uint32_t)__popc(need), curEnd - cur);
                if (!has && rank < n) {
                    ray_of(I.W, cur + rank - I.rayBase, I.W.order != 0, slot, k);
                    const DevCascade& C = I.W.C;
                    const float3 ro = probe_world_pos(C, (C.probeOffset + slot) % C.probeTotal);
                    const float3 rd = ray_dir(k, C.rays, I.W.P.frameJitter);
                    bestT = T_MAX;
                    tri = inst = -1;
                    bu = bv = 0.0f;
                    wide_begin<false>(I.W.S, w, ro, rd, bestT, tri, inst, bu, bv, vis, I.W.err);
                    has = true;
                }
                cur += n;
            }
        }
        if (!__any_sync(0xFFFFFFFFu, has)) {
            if (!more && pend == NONE && cur == curEnd) break;
            continue;
        }
        if (has) {
            const BatchItem& I = B.it[item];
            if (wide_step<false>(I.W.S, w, bestT, tri, inst, bu, bv, vis, I.W.err)) {
                wide_end<false>(I.W.S, w, bestT, tri, inst, bu, bv, vis, I.W.err);
                write_hit(I.W.C, slot, k, tri, inst, bestT, bu, bv);
                ++nRays;
                has = false;
            }
        }
    }
    add_visits(B.counters, 2, nRays, vis);
}

__global__ void __launch_bounds__(128) k_emit_batch(const __grid_constant__ BatchArgs B) {
    const uint32_t gg = blockIdx.x * blockDim.x + threadIdx.x;
    if (gg - (threadIdx.x & 31u) >= B.totalRays) return;  // whole warps only
    const BatchItem& I = B.it[batch_item(B, gg & ~31u)];
    if (!*I.W.S.valid) return;
    const uint32_t g = gg - I.rayBase;
    const uint32_t nJobs = emit_ray(I.W, g < I.rays, g, I.rayBase);
    if (B.counters) {
        const uint32_t warpDone = __reduce_add_sync(0xFFFFFFFFu, nJobs);
        if ((threadIdx.x & 31u) == 0 && warpDone) atomicAdd(&B.counters[1], (unsigned long long)warpDone);
    }
}

__global__ void __launch_bounds__(256, SB_SHADOW_MIN_BLOCKS) k_trace_shadow_batch(const __grid_constant__ BatchArgs B) {
    const BatchItem& I0 = B.it[0];
    const uint32_t total = min(*(volatile uint32_t*)&B.work[2], I0.W.jobCap);
    const uint32_t lane = threadIdx.x & 31u;
    Visits vis = {0, 0, 0, 0};
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&B.work[1], 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        uint32_t j = base + lane;
        if (j >= total) continue;
        const float4 a = I0.W.jobs[2 * j], b = I0.W.jobs[2 * j + 1];
        const uint32_t ray = __float_as_uint(b.w) >> 6;
        const BatchItem& I = B.it[batch_item(B, ray)];
        const bool pairs = any_pairs(I.W.S);
        shadow_job(I.W, pairs ? I.W.S.tlasPairs : I.W.S.tlas, pairs, a, b, ray - I.rayBase, vis);
    }
    add_visits(B.counters, 6, 0u, vis);
}

__global__ void __launch_bounds__(128) k_shade_batch(const __grid_constant__ BatchArgs B) {
    const uint32_t gg = blockIdx.x * blockDim.x + threadIdx.x;
    if (gg >= B.totalRays) return;
    const BatchItem& I = B.it[batch_item(B, gg & ~31u)];
    const uint32_t g = gg - I.rayBase;
    if (g >= I.rays || !*I.W.S.valid) return;
    shade_ray(I.W, g);
}

const void* trace_batch_kernel(int stage) {
    switch (stage) {
        case 0: return (const void*)k_trace_primary_batch;
        case 1: return (const void*)k_emit_batch;
        case 2: return (const void*)k_trace_shadow_batch;
        case 3: return (const void*)k_shade_batch;
        default: return nullptr;
    }
}

cudaError_t launch_trace_batch(const BatchArgs& B, const TraceTuning& tune, cudaStream_t st,
                               cudaEvent_t afterPrimary, cudaEvent_t afterShadow, cudaEvent_t afterClosest) {
    if (B.n == 0 || B.totalRays == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(B.work, 0, 3 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const int block = (int)tune.block;
    const uint32_t rays = B.totalRays;
    k_trace_primary_batch<<<persistent_grid((const void*)k_trace_primary_batch, block, 0, tune, rays), block, 0,
                            st>>>(B);
    note_launch();
    if (afterClosest) cudaEventRecord(afterClosest, st);
    k_emit_batch<<<(rays + 127) / 128, 128, 0, st>>>(B);
    note_launch();
    if (afterPrimary) cudaEventRecord(afterPrimary, st);
    k_trace_shadow_batch<<<persistent_grid((const void*)k_trace_shadow_batch, block, 0, tune, rays * 4u), block, 0,
                           st>>>(B);
    note_launch();
    if (afterShadow) cudaEventRecord(afterShadow, st);
    k_shade_batch<<<(rays + 127) / 128, 128, 0, st>>>(B);
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

namespace sb {
// The probe rays of a solve exactly as the trace stage forms them (probe
// origin and ray_dir with the current frame jitter): ray slot * rays + k.
__global__ void k_probe_rays(const DevCascade C, float jitter, float* ro, float* rd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.updatedCount * C.rays) return;
    const uint32_t slot = i / C.rays, k = i % C.rays;
    const float3 o = probe_world_pos(C, (C.probeOffset + slot) % C.probeTotal);
    const float3 d = ray_dir(k, C.rays, jitter);
    ro[3 * i] = o.x; ro[3 * i + 1] = o.y; ro[3 * i + 2] = o.z;
    rd[3 * i] = d.x; rd[3 * i + 1] = d.y; rd[3 * i + 2] = d.z;
}
// emitterVisKernel (gi_probes.js:2216-2260): per (updated probe, emitter) a
// shadow ray from the probe to a point of the emitter's disk, chosen by a sin
// hash of (probe, emitter, epoch seed) evaluated in separately rounded FP32,
// folded into the emitter's visibility history with retention 0.8.
__global__ void k_emitter_vis(DevScene S, DevCascade C, DevParams P, uint32_t* err) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t slot = gid / EMITTER_CAP, e = gid % EMITTER_CAP;
    if (slot >= C.updatedCount || e >= C.emitterCount || !*S.valid) return;
    const uint32_t probeIndex = (C.probeOffset + slot) % C.probeTotal;
    const float3 ro = probe_world_pos(C, probeIndex);
    const float* L = C.lights + (size_t)(C.emitterBase + e) * 17u;
    const float3 center = mk(L[1], L[2], L[3]);
    const float sourceRadius = fmaxf(L[14], 0.0f);
    const float3 axis = center - ro;
    const float dist = sqrtf(dot3(axis, axis));
    float sample = 0.0f;
    if (dist > fmaxf(sourceRadius, 1e-3f)) {
        const float3 d = axis * (1.0f / dist);
        const float3 up = fabsf(d.y) < 0.999f ? mk(0.0f, 1.0f, 0.0f) : mk(1.0f, 0.0f, 0.0f);
        const float3 tangent = normalize3(cross3(up, d));
        const float3 bitangent = cross3(d, tangent);
        const float seed = __fadd_rn(__fadd_rn(__fmul_rn(float(probeIndex), 12.9898f), __fmul_rn(float(e), 78.233f)),
                                     __fmul_rn(P.emitterVisSeed, 37.719f));
        const float h0 = __fmul_rn(sinf(seed), 43758.5453f);
        const float h1 = __fmul_rn(sinf(__fadd_rn(seed, 19.19f)), 24634.6345f);
        const float u = h0 - floorf(h0), v = h1 - floorf(h1);
        const float diskRadius = sqrtf(u) * sourceRadius;
        const float diskAngle = v * 6.283185307179586f;
        const float3 target = center + (tangent * (cosf(diskAngle) * diskRadius) + bitangent * (sinf(diskAngle) * diskRadius));
        const float3 sdir = normalize3(target - ro);
        const float traceBias = fmaxf(C.cellMin * 0.005f * P.debugTraceBiasScale, RAY_EPS * P.debugRayEpsScale);
        Visits vis = {0, 0, 0, 0};
        const bool pairs = any_pairs(S);
        const bool blocked = trace_any(S, pairs ? S.tlasPairs : S.tlas, ro, sdir,
                                       fmaxf(dist - sourceRadius - traceBias, 1e-4f), vis, err, pairs);
        sample = blocked ? 0.0f : 1.0f;
    }
    float* vp = C.emitterVis + (size_t)probeIndex * EMITTER_CAP + e;
    *vp = sample * (1.0f - EMITTER_VIS_RETENTION) + *vp * EMITTER_VIS_RETENTION;
}

cudaError_t launch_emitter_vis(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t* err,
                               cudaStream_t st) {
    const uint32_t n = C.updatedCount * EMITTER_CAP;
    if (n == 0 || C.emitterCount == 0) return cudaSuccess;
    k_emitter_vis<<<(n + 127) / 128, 128, 0, st>>>(S, C, P, err);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_probe_rays(const DevCascade& C, float jitter, float* ro, float* rd, cudaStream_t st) {
    const uint32_t n = C.updatedCount * C.rays;
    if (n == 0) return cudaSuccess;
    k_probe_rays<<<(n + 255) / 256, 256, 0, st>>>(C, jitter, ro, rd);
    note_launch();
    return cudaGetLastError();
}
}  // namespace sb

extern "C" uint32_t sb_triangle_test(void) { return SB_WATERTIGHT ? 1u : 0u; }
