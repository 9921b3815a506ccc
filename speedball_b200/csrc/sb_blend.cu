// sb_blend.cu — temporal blend of the probe histories and the RGBA16F atlas
// upload, fused into one kernel (blendKernel gi_probes.js:2317-2532 followed by
// uploadKernel 2737-2846: the upload's 3x3 filter only reads texels of the same
// probe tile, so one CTA per probe finishes both without a second launch).
// Also: the clustered light grid (lightGridKernel 1888-1938) and atlas clears
// (clearAtlasKernel 2690-2707).
#include "sb_math.cuh"
#include "sb_kernels.cuh"

namespace sb {

// One CTA blends BLEND_PROBES probes, one thread per (probe, interior texel).
// The cosine weight pow(max(dot(texelDir, rayDir), 0), cosPow) and the depth
// weight pow(cw, depthSharpness) depend on (texel, ray) only, not on the probe,
// so the CTA builds that 36 x rays table once in shared memory and every probe
// reuses it; per (texel, ray) the loop is then 9 FMA/ADD on shared operands.
// Per-ray features (radiance, luma, luma^2, hit distance, distance^2) are also
// formed once per ray instead of once per (texel, ray). Sums run in ray order
// in FP32 with per-texel Kahan compensation (kahan_fma), so each of the nine
// moments carries about 2 ulp of error whatever the ray count.
constexpr int BLEND_PROBES = 8;
constexpr int BLEND_TEXELS = OCT * OCT;
constexpr int BLEND_THREADS = BLEND_PROBES * BLEND_TEXELS;  // 288 = 9 warps

// ROUGH adds the rough reflection lobe (power 8, gi_probes.js:2388-2404): a
// third weight table, a coverage flag per ray and the blended rough history
// per texel; it stages 32 rays per pass so that the block stays within 48 KB.
template <bool ROUGH> struct BlendSmem {
    static constexpr int CH = ROUGH ? 32 : 64;  // rays staged per pass
    float4 texDir[BLEND_TEXELS];
    float4 rayDir[CH];
    float wc[CH][BLEND_TEXELS];               // cosine weight  [ray][texel]
    float wd[CH][BLEND_TEXELS];               // depth weight   [ray][texel]
    float wr[ROUGH ? CH : 1][BLEND_TEXELS];   // rough lobe weight cd^8
    union {
        struct {
            float4 fa[BLEND_PROBES][CH + 1];  // r, g, b, luma (row pad shifts banks)
            float4 fb[BLEND_PROBES][CH + 1];  // luma^2, dist, dist^2, reflection coverage (0 / 1)
        } f;
        float4 out[BLEND_PROBES][BLEND_TEXELS];        // filtered irradiance (after the sums)
    } u;
    float4 irr[BLEND_PROBES][BLEND_TEXELS];
    float2 dep[BLEND_PROBES][BLEND_TEXELS];
    float4 rough[ROUGH ? BLEND_PROBES : 1][BLEND_TEXELS];  // blended rough history
    float wsum[BLEND_TEXELS], dwsum[BLEND_TEXELS], swsum[BLEND_TEXELS];  // the same for every probe
};

// Blend + upload of probe slots [block * BLEND_PROBES, + BLEND_PROBES) of one
// solve; the body of the per-solve and the batched kernels.
template <bool ROUGH>
__device__ __forceinline__ void blend_upload_block(const DevCascade& C, const DevParams& P, uint32_t block,
                                                   BlendSmem<ROUGH>& S) {
    constexpr int CH = BlendSmem<ROUGH>::CH;
    const int tid = threadIdx.x;
    const int p = tid / BLEND_TEXELS, lane = tid % BLEND_TEXELS;
    const uint32_t base = block * BLEND_PROBES;
    const uint32_t slot = base + p;
    const bool live = slot < C.updatedCount;
    const uint32_t N = C.rays;
    const uint32_t nProbes = min((uint32_t)BLEND_PROBES, C.updatedCount - base);
    const float cosPow = fmaxf(P.debugCosinePower, 1e-4f);
    const bool cosUnit = cosPow == 1.0f;  // pow(x, 1) == x exactly
    const uint32_t sharpN = (uint32_t)P.depthSharpness;
    const bool sharpInt = P.depthSharpness >= 1.0f && P.depthSharpness <= 16.0f && float(sharpN) == P.depthSharpness;
    if (tid < BLEND_TEXELS) {
        float u = (float(tid % OCT) + 0.5f) / 6.0f, v = (float(tid / OCT) + 0.5f) / 6.0f;
        float3 d = oct_decode(u, v);
        S.texDir[tid] = make_float4(d.x, d.y, d.z, 0.0f);
    }

    float sr = 0.f, sg = 0.f, sb = 0.f, sl = 0.f, sl2 = 0.f, ws = 0.f, sd = 0.f, sd2 = 0.f, dws = 0.f;
    float cr = 0.f, cg = 0.f, cb = 0.f, cl = 0.f, cl2 = 0.f, cws = 0.f, cd = 0.f, cd2 = 0.f, cdw = 0.f;
    // rough lobe sums (sAcc, sHit, sWsum of gi_probes.js:2358-2360) and their compensations
    float xr = 0.f, xg = 0.f, xb = 0.f, xh = 0.f, xws = 0.f;
    float kxr = 0.f, kxg = 0.f, kxb = 0.f, kxh = 0.f, kxws = 0.f;
    // a true miss feeds the lobe only with an explicit sky fallback (gi_probes.js:2364-2367)
    const float skyValid = ROUGH ? P.reflectionSkyFallback * P.skyConfigured * (P.skyIntensity > 0.0f ? 1.0f : 0.0f)
                                 : 0.0f;
    for (uint32_t c = 0; c < N; c += CH) {
        const uint32_t n = min((uint32_t)CH, N - c);
        __syncthreads();  // previous pass done with the table and features
        for (uint32_t e = tid; e < nProbes * n; e += BLEND_THREADS) {
            uint32_t q = e / n, k = e % n;
            float4 r = C.rayData[(size_t)(base + q) * N + c + k];
            float rl = luma3(mk(r.x, r.y, r.z));
            float hitT = r.w;
            float decoded = hitT < -1.5f ? -hitT - 2.0f : hitT;
            float rdist = hitT == -1.0f ? C.maxDist : decoded;
            S.u.f.fa[q][k] = make_float4(r.x, r.y, r.z, rl);
            // local hits count, a miss counts with the sky fallback, encoded unshaded hits never
            const float valid = hitT >= 0.0f ? 1.0f : (hitT == -1.0f ? skyValid : 0.0f);
            S.u.f.fb[q][k] = make_float4(rl * rl, rdist, rdist * rdist, valid);
        }
        if ((uint32_t)tid < n) {
            float3 d = ray_dir(c + tid, N, P.frameJitter);
            S.rayDir[tid] = make_float4(d.x, d.y, d.z, 0.0f);
        }
        __syncthreads();
        for (uint32_t e = tid; e < n * BLEND_TEXELS; e += BLEND_THREADS) {
            uint32_t k = e / BLEND_TEXELS, j = e % BLEND_TEXELS;
            float4 a = S.texDir[j], b = S.rayDir[k];
            float cd = fmaxf(a.x * b.x + a.y * b.y + a.z * b.z, 0.0f);
            float cw = cosUnit ? cd : powf(cd, cosPow);
            float dw;
            if (sharpInt) {  // small integer exponent: square-and-multiply (a few ulp of powf)
                dw = 1.0f;
                float x = cw;
                for (uint32_t m = sharpN; m; m >>= 1) {
                    if (m & 1u) dw *= x;
                    x *= x;
                }
            } else {
                dw = powf(cw, P.depthSharpness);
            }
            S.wc[k][j] = cw;
            S.wd[k][j] = dw;
            if (ROUGH) {  // fixed power-8 lobe as ((cd^2)^2)^2 (gi_probes.js:2389-2393)
                const float c2 = cd * cd, c4 = c2 * c2;
                S.wr[k][j] = c4 * c4;
            }
        }
        __syncthreads();
        if (live) {
#pragma unroll 4
            for (uint32_t k = 0; k < n; ++k) {
                float w = S.wc[k][lane], v = S.wd[k][lane];
                float4 a = S.u.f.fa[p][k], b = S.u.f.fb[p][k];
                kahan_fma(sr, cr, w, a.x);
                kahan_fma(sg, cg, w, a.y);
                kahan_fma(sb, cb, w, a.z);
                kahan_fma(sl, cl, w, a.w);
                kahan_fma(sl2, cl2, w, b.x);
                kahan_fma(sd, cd, v, b.y);
                kahan_fma(sd2, cd2, v, b.z);
                if (ROUGH) {
                    const float r = S.wr[k][lane];
                    const float rv = r * b.w;  // coverage is 0 or 1: exact
                    kahan_fma(xr, kxr, rv, a.x);
                    kahan_fma(xg, kxg, rv, a.y);
                    kahan_fma(xb, kxb, rv, a.z);
                    kahan_fma(xh, kxh, rv, 1.0f);
                }
            }
            if (p == 0)  // the weight sums depend on (texel, ray) only: the first probe's lanes form them
                for (uint32_t k = 0; k < n; ++k) {
                    kahan_fma(ws, cws, S.wc[k][lane], 1.0f);
                    kahan_fma(dws, cdw, S.wd[k][lane], 1.0f);
                    if (ROUGH) kahan_fma(xws, kxws, S.wr[k][lane], 1.0f);
                }
        }
    }
    if (p == 0) {
        S.wsum[lane] = ws;
        S.dwsum[lane] = dws;
        S.swsum[lane] = xws;
    }
    __syncthreads();  // features no longer read: S.u.out may be written; weight sums published
    ws = S.wsum[lane];
    dws = S.dwsum[lane];
    xws = S.swsum[lane];

    const uint32_t probeIndex = live ? (C.probeOffset + slot) % C.probeTotal : 0u;
    if (live && C.emitterCount) {
        // injectEmitterVirtualRays (gi_probes.js:2262-2310): each emitter as
        // kVirtual = min(N, N Omega / 4 pi) rays toward its centre carrying its
        // radiance x visibility, Omega = min(2 pi, projectedArea / d^2)
        const float3 ro = probe_world_pos(C, probeIndex);
        const float4 td = S.texDir[lane];
        for (uint32_t e = 0; e < C.emitterCount; ++e) {
            const float* L = C.lights + (size_t)(C.emitterBase + e) * 17u;
            const float3 axis = mk(L[1], L[2], L[3]) - ro;
            const float dist = sqrtf(dot3(axis, axis));
            if (!(dist > fmaxf(fmaxf(L[14], 0.0f), 1e-3f))) continue;
            const float3 d = axis * (1.0f / dist);
            const float omega = fminf(6.283185307179586f, fmaxf(L[15], 0.0f) / (dist * dist));
            const float kVirtual = fminf(float(N), float(N) * omega / 12.566370614359172f);
            const float vis = C.emitterVis[(size_t)probeIndex * EMITTER_CAP + e];
            const float3 Lc = mk(L[7] * vis, L[8] * vis, L[9] * vis);
            const float cdot = fmaxf(td.x * d.x + td.y * d.y + td.z * d.z, 0.0f);
            const float wk = (cosUnit ? cdot : powf(cdot, cosPow)) * kVirtual;
            const float lum = luma3(Lc);
            kahan_fma(sr, cr, wk, Lc.x);
            kahan_fma(sg, cg, wk, Lc.y);
            kahan_fma(sb, cb, wk, Lc.z);
            kahan_fma(sl, cl, wk, lum);
            kahan_fma(sl2, cl2, wk, lum * lum);
            ws += wk;
            if (ROUGH) {  // the secondary (power-8) weight of the same virtual rays
                const float c2 = cdot * cdot, c4 = c2 * c2;
                const float sk = c4 * c4 * kVirtual;
                kahan_fma(xr, kxr, sk, Lc.x);
                kahan_fma(xg, kxg, sk, Lc.y);
                kahan_fma(xb, kxb, sk, Lc.z);
                kahan_fma(xh, kxh, sk, 1.0f);
                xws += sk;
            }
        }
    }
    if (live) {
        const uint32_t lx = lane % OCT + BORDER, ly = lane / OCT + BORDER;
        const uint32_t local = ly * TILE + lx;
        float wden = fmaxf(ws, 1e-4f);
        float3 meanRad = mk(sr / wden, sg / wden, sb / wden);
        float curL = sl / wden, curM2 = sl2 / wden;
        float dden = fmaxf(dws, 1e-4f);
        float meanR = sd / dden, meanR2 = sd2 / dden;

        const size_t ib = (size_t)probeIndex * 64u + local;
        float4 prev4 = C.irr[ib];
        float3 prev = xyz(prev4);
        bool wasBlack = (prev.x + prev.y + prev.z) < 1e-6f;
        float prevL = luma3(prev);
        float prevM2 = prev4.w;
        float prevVar = fmaxf(prevM2 - prevL * prevL, 0.0f);
        float curVar = fmaxf(curM2 - curL * curL, 0.0f);
        float lumRef = fmaxf(fmaxf(curL, prevL), 0.0f);
        float varFloor = P.debugTempVarEps + lumRef * lumRef * P.debugTempVarRel;
        float sigma = sqrtf(prevVar + curVar + varFloor);
        float absDelta = fabsf(curL - prevL);
        float s0 = sigma * P.debugTempChangeSigma0;
        float s1 = sigma * fmaxf(P.tempChangeSigma1, P.debugTempChangeSigma0 + 0.01f);
        float changeW = clampf((absDelta - s0) / fmaxf(s1 - s0, 1e-6f), 0.0f, 1.0f);
        float H = P.hysteresis;
        float rawNoiseH = H + (1.0f - H) * P.debugTempNoiseHBoost;
        float rawChangeH = fmaxf(H - P.tempChangeHDrop, P.debugTempMinChangeH);
        float rawHEff = mixf(rawNoiseH, rawChangeH, changeW);
        float hEff = powf(clampf(rawHEff, 1e-6f, 1.0f), P.hysteresisExponent);
        float h = wasBlack ? 0.0f : hEff;
        float band = sqrtf(prevVar + varFloor) * P.tempClampSigma;
        float clampScale = fminf(1.0f, band / fmaxf(absDelta, 1e-6f));
        float3 clipped = prev + (meanRad - prev) * clampScale;
        float3 cand = wasBlack ? meanRad : clipped;
        float3 blended = mk(mixf(cand.x, prev.x, h), mixf(cand.y, prev.y, h), mixf(cand.z, prev.z, h));
        float m2 = mixf(curM2, prevM2, h);
        float4 outIrr = make_float4(blended.x, blended.y, blended.z, m2);
        C.irr[ib] = outIrr;

        float2 dprev = C.depth[ib];
        bool dWasZero = dprev.x < 1e-6f;
        if (ROUGH) {
            // rough history (gi_probes.js:2505-2522): the steady / noisy reference retention,
            // independent of the diffuse change detector; seeded where depth is unseeded
            const float sDen = fmaxf(xws, 1e-4f);
            const float4 sCur = make_float4(xr / sDen, xg / sDen, xb / sDen, clampf(xh / sDen, 0.0f, 1.0f));
            const float steadyH = powf(clampf(rawNoiseH, 1e-6f, 1.0f), P.hysteresisExponent);
            const float sh = dWasZero ? 0.0f : steadyH;
            const float4 sPrev = C.roughSpec[ib];
            const float4 sOut = make_float4(mixf(sCur.x, sPrev.x, sh), mixf(sCur.y, sPrev.y, sh),
                                            mixf(sCur.z, sPrev.z, sh), mixf(sCur.w, sPrev.w, sh));
            C.roughSpec[ib] = sOut;
            S.rough[p][lane] = sOut;
        }
        float rawDepthH = clampf(H * P.debugDepthHistoryScale, 0.0f, 0.999f);
        float depthH = powf(fmaxf(rawDepthH, 1e-6f), P.hysteresisExponent);
        float dh = dWasZero ? 0.0f : depthH;
        float2 outDep = make_float2(mixf(meanR, dprev.x, dh), mixf(meanR2, dprev.y, dh));
        C.depth[ib] = outDep;
        S.irr[p][lane] = outIrr;
        S.dep[p][lane] = outDep;
    }
    __syncthreads();

    // upload: 3x3 bilateral filter of the new history (reads this tile only)
    if (live) {
        const int sx = (int)(lane % OCT), sy = (int)(lane / OCT);
        float4 c4 = S.irr[p][lane];
        float3 eC = xyz(c4);
        float lumaC = luma3(eC);
        float varC = fmaxf(c4.w - lumaC * lumaC, 0.0f);
        float smW = 1.0f + P.filterSmooth * 6.0f;
        float kEff = 8.0f * smW * P.debugFilterKScale;
        float relEff = 0.0225f * smW * P.debugFilterRelScale;
        float den = fmaxf(varC * kEff + fmaxf(0.001f * P.debugFilterEpsScale, lumaC * lumaC * relEff), 1e-8f);
        float3 facc = mk(0.f, 0.f, 0.f);
        float fw = 0.0f;
#pragma unroll
        for (int jy = -1; jy <= 1; ++jy)
#pragma unroll
            for (int jx = -1; jx <= 1; ++jx) {
                const float gw = (jx == 0 && jy == 0) ? 1.0f
                                 : (jx == 0 || jy == 0) ? 0.6065306597126334f   // exp(-0.5)
                                                        : 0.36787944117144233f; // exp(-1)
                int nx = min(max(sx + jx, 0), OCT - 1), ny = min(max(sy + jy, 0), OCT - 1);
                float3 en = xyz(S.irr[p][ny * OCT + nx]);
                float dl = luma3(en) - lumaC;
                float es = expf(dl * dl / den * -1.0f);
                float w = gw * es;
                facc = facc + en * w;
                fw += w;
            }
        float fden = fmaxf(fw, 1e-4f);
        float3 filt = mk(facc.x / fden, facc.y / fden, facc.z / fden);
        float s = P.filterStrength;
        S.u.out[p][lane] = make_float4(mixf(eC.x, filt.x, s), mixf(eC.y, filt.y, s), mixf(eC.z, filt.z, s), 1.0f);
        if (C.eOut) C.eOut[(size_t)probeIndex * BLEND_TEXELS + lane] = S.u.out[p][lane];  // pre-FP16 value
    }
    __syncthreads();

    // 64 texels per probe: interior + canonical mirrored gutter (gi_probes.js:2816-2839)
    for (uint32_t e = tid; e < nProbes * 64u; e += BLEND_THREADS) {
        const uint32_t q = e / 64u, texel = e % 64u;
        const uint32_t probeIndex = (C.probeOffset + base + q) % C.probeTotal;
        const int edge = TILE - 1, lo = BORDER, hi = BORDER + OCT - 1;
        int lx = (int)(texel % TILE), ly = (int)(texel / TILE);
        bool onLeft = lx == 0, onRight = lx == edge, onTop = ly == 0, onBottom = ly == edge;
        bool colB = onLeft || onRight, rowB = onTop || onBottom, corner = colB && rowB;
        int sx = corner ? (onLeft ? hi : lo) : (rowB ? edge - lx : (colB ? (onLeft ? lo : hi) : lx));
        int sy = corner ? (onTop ? hi : lo) : (rowB ? (onTop ? lo : hi) : (colB ? edge - ly : ly));
        int src = (sy - BORDER) * OCT + (sx - BORDER);
        uint32_t col = probeIndex % C.res[0];
        uint32_t row = (probeIndex / (C.res[0] * C.res[1])) * C.res[1] + (probeIndex / C.res[0]) % C.res[1];
        size_t t = (size_t)(row * TILE + ly) * C.atlasW + col * TILE + lx;
        C.atlas[t] = float4_to_half4(S.u.out[q][src]);
        float2 d = S.dep[q][src];
        C.depthAtlas[t] = float4_to_half4(make_float4(d.x, d.y, 0.0f, 1.0f));
        if (ROUGH) C.roughAtlas[t] = float4_to_half4(S.rough[q][src]);  // unfiltered (gi_probes.js:2789-2795, 2841-2843)
    }
}

template <bool ROUGH>
__global__ void __launch_bounds__(BLEND_THREADS) k_blend_upload(DevCascade C, DevParams P) {
    __shared__ BlendSmem<ROUGH> S;
    blend_upload_block<ROUGH>(C, P, blockIdx.x, S);
}

// Every item of a batch: CTAs [blendBase, blendBase + blendBlocks) belong to item i.
__global__ void __launch_bounds__(BLEND_THREADS) k_blend_upload_batch(const __grid_constant__ BatchArgs B) {
    __shared__ BlendSmem<false> S;  // batches carry no reflection lobes
    uint32_t i = 0;
    while (i + 1 < B.n && blockIdx.x >= B.it[i + 1].blendBase) ++i;
    const BatchItem& I = B.it[i];
    if (blockIdx.x - I.blendBase >= I.blendBlocks) return;
    blend_upload_block<false>(I.W.C, I.W.P, blockIdx.x - I.blendBase, S);
}

cudaError_t launch_blend_upload(const DevCascade& C, const DevParams& P, cudaStream_t st) {
    if (C.updatedCount == 0) return cudaSuccess;
    const uint32_t blocks = (C.updatedCount + BLEND_PROBES - 1) / BLEND_PROBES;
    if (C.reflect && C.roughSpec)
        k_blend_upload<true><<<blocks, BLEND_THREADS, 0, st>>>(C, P);
    else
        k_blend_upload<false><<<blocks, BLEND_THREADS, 0, st>>>(C, P);
    note_launch();
    return cudaGetLastError();
}

const void* blend_batch_kernel() { return (const void*)k_blend_upload_batch; }

cudaError_t launch_blend_upload_batch(const BatchArgs& B, cudaStream_t st) {
    if (B.n == 0 || B.blendBlocks == 0) return cudaSuccess;
    k_blend_upload_batch<<<B.blendBlocks, BLEND_THREADS, 0, st>>>(B); note_launch();
    return cudaGetLastError();
}

uint32_t blend_blocks(uint32_t updatedCount) { return (updatedCount + BLEND_PROBES - 1) / BLEND_PROBES; }

// glossyKernel (gi_probes.js:2538-2686): the power-64 lobe on the glossy tiles
// (glossyOct^2 texels + a one-texel mirrored gutter). Tier high resolves the
// texels with local % 2 == glossyPhase, ultra every texel. Each texel keeps a
// per-ray-mean numerator (rgb, coverage) and support in its history, blended
// with one retention, and stores their ratio to the glossy atlas.
//
// The weight pow(max(dot(texelDir, rayDir), 0), 64) depends on (texel, ray)
// only, so one CTA serves GLOSSY_PROBES probes: a thread owns one resolved
// texel, forms each ray's weight once and applies it to every probe's ray
// (four FMA per probe and ray, on radiance premultiplied by coverage). The
// terms are non-negative, so plain FP32 sums of at most 256 rays stay within
// 256 ulp of the exact sum. A CTA holds `groups` such thread groups (each its
// own GLOSSY_PROBES probes) when a group is small (tier high: 50 resolved
// texels), as far as the staged rays fit 48 KB. Measured on the atrium (4,096
// probes x 64 rays): tier ultra 0.127 ms with one probe per CTA, 0.084 ms with
// 8 probes per thread, 0.069 ms (ncu) with 4 and the higher occupancy.
constexpr uint32_t GLOSSY_PROBES = 4;
constexpr uint32_t GLOSSY_MAX_RAYS = 256;  // raysPerProbe <= 256 (gi_probes.js:988-992)

__device__ __forceinline__ float pow64(float c) {
    const float c2 = c * c, c4 = c2 * c2, c8 = c4 * c4, c16 = c8 * c8, c32 = c16 * c16;
    return c32 * c32;
}

__global__ void __launch_bounds__(352) k_glossy(DevCascade C, DevParams P, uint32_t groupThreads) {
    extern __shared__ float4 gsm[];
    const uint32_t N = C.rays;
    const uint32_t groups = blockDim.x / groupThreads;
    float4* dir = gsm;  // N ray directions, then groups x GLOSSY_PROBES x N rays: rgb, coverage
    const uint32_t cbase = blockIdx.x * groups * GLOSSY_PROBES;
    const uint32_t cProbes = min(groups * GLOSSY_PROBES, C.updatedCount - cbase);
    const float skyValid = P.reflectionSkyFallback * P.skyConfigured * (P.skyIntensity > 0.0f ? 1.0f : 0.0f);
    for (uint32_t k = threadIdx.x; k < N; k += blockDim.x) {
        const float3 d = ray_dir(k, N, P.frameJitter);
        dir[k] = make_float4(d.x, d.y, d.z, 0.0f);
    }
    for (uint32_t e = threadIdx.x; e < groups * GLOSSY_PROBES * N; e += blockDim.x) {
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // slots past the last probe stay zero
        if (e < cProbes * N) {  // radiance x coverage, coverage (0 or 1: the products are exact)
            const float4 r = C.rayData[(size_t)cbase * N + e];
            const float valid = r.w >= 0.0f ? 1.0f : (r.w == -1.0f ? skyValid : 0.0f);
            v = make_float4(r.x * valid, r.y * valid, r.z * valid, valid);
        }
        gsm[N + e] = v;
    }
    __syncthreads();
    const uint32_t group = threadIdx.x / groupThreads;
    const uint32_t base = cbase + group * GLOSSY_PROBES;
    if (base >= C.updatedCount) return;
    const uint32_t nProbes = min(GLOSSY_PROBES, C.updatedCount - base);
    const float4* rad = gsm + N + (size_t)group * GLOSSY_PROBES * N;  // this group's probes
    const uint32_t tile = C.glossyTile, oct = C.glossyOct, texels = tile * tile;
    const uint32_t step = C.glossyInterval > 1u ? C.glossyInterval : 1u;
    const uint32_t local = (threadIdx.x % groupThreads) * step + (step > 1u ? C.glossyPhase : 0u);
    // lanes past the last texel run the ray loop with zero weights and store nothing
    const bool active = local < texels;
    const int lx = (int)(local % tile), ly = (int)(local / tile);
    // canonical mirrored gutter, resolved before the direction (gi_probes.js:2571-2593)
    const int edge = (int)tile - 1, lo = BORDER, hi = BORDER + (int)oct - 1;
    const bool onLeft = lx == 0, onRight = lx == edge, onTop = ly == 0, onBottom = ly == edge;
    const bool colB = onLeft || onRight, rowB = onTop || onBottom, corner = colB && rowB;
    const int sx = corner ? (onLeft ? hi : lo) : (rowB ? edge - lx : (colB ? (onLeft ? lo : hi) : lx));
    const int sy = corner ? (onTop ? hi : lo) : (rowB ? (onTop ? lo : hi) : (colB ? edge - ly : ly));
    const float3 td = active ? oct_decode((float(sx - BORDER) + 0.5f) / float(oct),
                                          (float(sy - BORDER) + 0.5f) / float(oct))
                             : mk(0.0f, 0.0f, 0.0f);
    float ar[GLOSSY_PROBES], ag[GLOSSY_PROBES], ab[GLOSSY_PROBES], ah[GLOSSY_PROBES];
#pragma unroll
    for (uint32_t q = 0; q < GLOSSY_PROBES; ++q) ar[q] = ag[q] = ab[q] = ah[q] = 0.0f;
    float aw = 0.0f;
    // every group slot is accumulated (a short last group's extra slots hold zero
    // rays whose sums are never stored): no branch in the loop
#pragma unroll 2
    for (uint32_t k = 0; k < N; ++k) {
        const float4 d = dir[k];
        const float gw = pow64(fmaxf(td.x * d.x + td.y * d.y + td.z * d.z, 0.0f));
        aw += gw;
#pragma unroll
        for (uint32_t q = 0; q < GLOSSY_PROBES; ++q) {
            const float4 r = rad[q * N + k];
            ar[q] = fmaf(gw, r.x, ar[q]);
            ag[q] = fmaf(gw, r.y, ag[q]);
            ab[q] = fmaf(gw, r.z, ab[q]);
            ah[q] = fmaf(gw, r.w, ah[q]);
        }
    }
    if (!active) return;
    const float invRays = 1.0f / float(N);  // equals float(1 / N) for every allowed N
    const float H = P.hysteresis;
    const float refH = H + (1.0f - H) * P.debugTempNoiseHBoost;
    const float glossyH = powf(clampf(refH, 1e-6f, 1.0f), P.hysteresisExponent * float(C.glossyInterval));
#pragma unroll
    for (uint32_t q = 0; q < GLOSSY_PROBES; ++q) {
        if (q >= nProbes) break;
        const uint32_t probeIndex = (C.probeOffset + base + q) % C.probeTotal;
        float r = ar[q], g = ag[q], b = ab[q], h = ah[q], w = aw;
        // the emitters' virtual rays with the power-64 weight (gi_probes.js:2624-2638)
        if (C.emitterCount) {
            const float3 ro = probe_world_pos(C, probeIndex);
            for (uint32_t e = 0; e < C.emitterCount; ++e) {
                const float* L = C.lights + (size_t)(C.emitterBase + e) * 17u;
                const float3 axis = mk(L[1], L[2], L[3]) - ro;
                const float dist = sqrtf(dot3(axis, axis));
                if (!(dist > fmaxf(fmaxf(L[14], 0.0f), 1e-3f))) continue;
                const float3 dd = axis * (1.0f / dist);
                const float omega = fminf(6.283185307179586f, fmaxf(L[15], 0.0f) / (dist * dist));
                const float kVirtual = fminf(float(N), float(N) * omega / 12.566370614359172f);
                const float vis = C.emitterVis[(size_t)probeIndex * EMITTER_CAP + e];
                const float wk = pow64(fmaxf(td.x * dd.x + td.y * dd.y + td.z * dd.z, 0.0f)) * kVirtual;
                r = fmaf(wk, L[7] * vis, r);
                g = fmaf(wk, L[8] * vis, g);
                b = fmaf(wk, L[9] * vis, b);
                h += wk;
                w += wk;
            }
        }
        // numerator / support history (gi_probes.js:2640-2674)
        const size_t gt = (size_t)probeIndex * texels + local;
        const float4 prevNum = C.glossyNum[gt];
        const float prevDen = C.glossyDen[gt];
        const float gh = prevDen < 1e-6f ? 0.0f : glossyH;
        const float4 num = make_float4(mixf(r * invRays, prevNum.x, gh), mixf(g * invRays, prevNum.y, gh),
                                       mixf(b * invRays, prevNum.z, gh), mixf(h * invRays, prevNum.w, gh));
        const float den = fmaxf(mixf(w * invRays, prevDen, gh), 1e-6f);
        C.glossyNum[gt] = num;
        C.glossyDen[gt] = den;
        const uint32_t col = probeIndex % C.glossyTilesX, row = probeIndex / C.glossyTilesX;
        const size_t t = (size_t)(row * tile + (uint32_t)ly) * C.glossyAtlasW + col * tile + (uint32_t)lx;
        C.glossyAtlas[t] = float4_to_half4(make_float4(num.x / den, num.y / den, num.z / den,
                                                       clampf(num.w / den, 0.0f, 1.0f)));
    }
}

cudaError_t launch_glossy(const DevCascade& C, const DevParams& P, cudaStream_t st) {
    if (C.updatedCount == 0 || !C.glossyNum || C.glossyInterval == 0 || C.rays > GLOSSY_MAX_RAYS)
        return cudaSuccess;
    const uint32_t texels = C.glossyTile * C.glossyTile;
    const uint32_t active = (texels + C.glossyInterval - 1u) / C.glossyInterval;  // one thread per resolved texel
    const uint32_t groupThreads = (active + 31u) / 32u * 32u;
    if (groupThreads > 352u) return cudaErrorInvalidConfiguration;
    // groups per CTA: up to 256 threads, the staged rays within 48 KB
    uint32_t groups = 1;
    while (groups < 4 && (groups + 1) * groupThreads <= 256u &&
           (size_t)C.rays * (1u + (groups + 1) * GLOSSY_PROBES) * sizeof(float4) <= 48u * 1024u)
        ++groups;
    const size_t smem = (size_t)C.rays * (1u + groups * GLOSSY_PROBES) * sizeof(float4);
    const uint32_t perCta = groups * GLOSSY_PROBES;
    const uint32_t blocks = (C.updatedCount + perCta - 1u) / perCta;
    k_glossy<<<blocks, groups * groupThreads, smem, st>>>(C, P, groupThreads); note_launch();
    return cudaGetLastError();
}

// lightGridKernel, gi_probes.js:1893-1937. Every operation is separately
// rounded (no contraction) so the lists match an FP32 evaluation exactly.
// The gate fields of the 64 light records (17 floats each, not 16-byte
// aligned) as three float4 per light, so the emission stage reads a light's
// gates with three vector loads: (position, range), (direction, type),
// (colour, emitter class) = record fields (1-3, 10), (4-6, 0), (7-9, 16).
__global__ void k_light_gates(const float* lights, float4* gates) {
    const uint32_t i = threadIdx.x;
    if (i >= 64u) return;
    const float* L = lights + i * 17u;
    gates[3 * i] = make_float4(L[1], L[2], L[3], L[10]);
    gates[3 * i + 1] = make_float4(L[4], L[5], L[6], L[0]);
    gates[3 * i + 2] = make_float4(L[7], L[8], L[9], L[16]);
}

cudaError_t launch_light_gates(const float* lights, float4* gates, cudaStream_t st) {
    k_light_gates<<<1, 64, 0, st>>>(lights, gates);
    note_launch();
    return cudaGetLastError();
}

__global__ void k_light_grid(float* lights, uint32_t lightCount, DevCascade g0, uint32_t cells) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    uint32_t cellsX = g0.res[0] - 1u, cellsY = g0.res[1] - 1u, cellsZ = g0.res[2] - 1u;
    uint32_t ix = c % cellsX, iy = (c / cellsX) % cellsY, iz = c / (cellsX * cellsY);
    float csx = __fdiv_rn(g0.gridSize[0], float(cellsX));
    float csy = __fdiv_rn(g0.gridSize[1], float(cellsY));
    float csz = __fdiv_rn(g0.gridSize[2], float(cellsZ));
    float mnx = __fadd_rn(g0.gridMin[0], __fmul_rn(float(ix), csx));
    float mny = __fadd_rn(g0.gridMin[1], __fmul_rn(float(iy), csy));
    float mnz = __fadd_rn(g0.gridMin[2], __fmul_rn(float(iz), csz));
    float mxx = __fadd_rn(mnx, csx), mxy = __fadd_rn(mny, csy), mxz = __fadd_rn(mnz, csz);
    float* list = lights + LIGHT_DATA + c * 17u;
    uint32_t count = 0;
    for (uint32_t li = 0; li < lightCount; ++li) {
        const float* L = lights + li * 17u;
        float ltype = L[0], px = L[1], py = L[2], pz = L[3], lrange = L[10];
        float dx = fmaxf(fmaxf(__fsub_rn(mnx, px), 0.0f), __fsub_rn(px, mxx));
        float dy = fmaxf(fmaxf(__fsub_rn(mny, py), 0.0f), __fsub_rn(py, mxy));
        float dz = fmaxf(fmaxf(__fsub_rn(mnz, pz), 0.0f), __fsub_rn(pz, mxz));
        float padded = __fadd_rn(lrange, fmaxf(1e-4f, __fmul_rn(lrange, 1e-5f)));
        float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        bool intersects = d2 <= __fmul_rn(padded, padded);
        bool member = ltype < 2.5f && (ltype < 0.5f || lrange <= 0.0f || intersects);
        if (member) {
            if (count < 16u) list[1 + count] = float(li);
            count++;
        }
    }
    list[0] = float(count > 16u ? 17u : count);
}

cudaError_t launch_light_grid(float* lights, uint32_t lightCount, const DevCascade& g0, cudaStream_t st) {
    uint32_t cells = (g0.res[0] - 1u) * (g0.res[1] - 1u) * (g0.res[2] - 1u);
    if (cells == 0) return cudaSuccess;
    k_light_grid<<<(cells + 127) / 128, 128, 0, st>>>(lights, lightCount, g0, cells); note_launch();
    return cudaGetLastError();
}

// clearAtlasKernel, gi_probes.js:2690-2707: atlases to (0,0,0,1); histories to 0.
__global__ void k_clear_cascade(DevCascade C) {
    size_t n = (size_t)C.atlasW * C.atlasH;
    size_t h = (size_t)C.probeTotal * 64u;
    uint2 v = float4_to_half4(make_float4(0.f, 0.f, 0.f, 1.f));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n || i < h; i += (size_t)gridDim.x * blockDim.x) {
        if (i < n) { C.atlas[i] = v; C.depthAtlas[i] = v; }
        if (i < h) { C.irr[i] = make_float4(0.f, 0.f, 0.f, 0.f); C.depth[i] = make_float2(0.f, 0.f); }
    }
}

cudaError_t launch_clear_cascade(const DevCascade& C, cudaStream_t st) {
    k_clear_cascade<<<148 * 4, 256, 0, st>>>(C); note_launch();
    return cudaGetLastError();
}

}  // namespace sb
