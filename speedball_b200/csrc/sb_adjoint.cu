// sb_adjoint.cu — reverse pass of shade + blend + upload for a differentiable
// solve sequence (sb_forward_record / sb_backward). Hit records and shadow
// visibility are inputs recorded by the forward, so only the shading is
// re-evaluated; every branch the forward took (wasBlack, clamps, max/min
// selects) is held at the side the forward value chose. The RGBA16F rounding
// of the atlas that feeds the next solve's bounce read is passed straight
// through (the gradient of a texel is the gradient of its FP32 source).
//
// Stages, per solve s from the last back to the first:
//   k_upload_bwd  dL/dE of the 36 interior texels (plus the gutter copies'
//                 share of dL/dAtlas) -> dL/dH through the 3x3 bilateral filter
//                 (uploadKernel, gi_probes.js:2737-2846).
//   k_blend_bwd   dL/dH(s+1) -> dL/d(ray radiance) and dL/dH(s) through the
//                 cosine-weighted moments and the temporal clamp / hysteresis
//                 mix (blendKernel, gi_probes.js:2317-2532).
//   k_shade_bwd   dL/d(ray radiance) -> material albedo / emissive, light scale
//                 and dL/dAtlas(s) through the NEE terms and the bounce read
//                 (traceKernel shading, gi_probes.js:2020-2206).
#include "sb_wave.cuh"
#include "sb_kernels.cuh"

namespace sb {

namespace {

constexpr float LW_R = 0.2126f, LW_G = 0.7152f, LW_B = 0.0722f;  // luma3 weights

__device__ __forceinline__ float3 lumaw3(float s) { return mk(LW_R * s, LW_G * s, LW_B * s); }

__device__ __forceinline__ void sh_add3(float* p, float3 v) {
    atomicAdd(p, v.x);
    atomicAdd(p + 1, v.y);
    atomicAdd(p + 2, v.z);
}

// Interior texel j (0..35) of a probe -> its index in the 8x8 history tile.
__device__ __forceinline__ uint32_t interior_local(uint32_t j) { return (j / OCT + BORDER) * TILE + j % OCT + BORDER; }

// Atlas texel (lx, ly) of probe p's 8x8 tile.
__device__ __forceinline__ size_t tile_texel(const DevCascade& C, uint32_t p, uint32_t lx, uint32_t ly) {
    uint32_t col = p % C.res[0];
    uint32_t row = (p / (C.res[0] * C.res[1])) * C.res[1] + (p / C.res[0]) % C.res[1];
    return (size_t)(row * TILE + ly) * C.atlasW + col * TILE + lx;
}

// Interior lane that tile texel (lx, ly) copies (the mirrored gutter,
// gi_probes.js:2816-2839).
__device__ __forceinline__ uint32_t gutter_source(uint32_t lx, uint32_t ly) {
    const int edge = TILE - 1, lo = BORDER, hi = BORDER + OCT - 1;
    bool onLeft = lx == 0, onRight = lx == (uint32_t)edge, onTop = ly == 0, onBottom = ly == (uint32_t)edge;
    bool colB = onLeft || onRight, rowB = onTop || onBottom, corner = colB && rowB;
    int sx = corner ? (onLeft ? hi : lo) : (rowB ? edge - (int)lx : (colB ? (onLeft ? lo : hi) : (int)lx));
    int sy = corner ? (onTop ? hi : lo) : (rowB ? (onTop ? lo : hi) : (colB ? edge - (int)ly : (int)ly));
    return (uint32_t)((sy - BORDER) * OCT + (sx - BORDER));
}

}  // namespace

// ---------------------------------------------------------------- loss

__global__ void __launch_bounds__(256) k_adjoint_loss(const float4* E, const float* target, uint32_t n, float4* gE,
                                                      double* loss) {
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 e = E[i];
        float dx = e.x - target[3 * i], dy = e.y - target[3 * i + 1], dz = e.z - target[3 * i + 2];
        gE[i] = make_float4(2.0f * dx, 2.0f * dy, 2.0f * dz, 0.0f);
        acc += (double)dx * dx + (double)dy * dy + (double)dz * dz;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(loss, s);
    }
}

cudaError_t launch_adjoint_loss(const float4* E, const float* target, uint32_t n, float4* gE, double* loss,
                                cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(double), st);
    if (e != cudaSuccess || n == 0) return e;
    uint32_t blocks = (n + 255) / 256;
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    k_adjoint_loss<<<blocks, 256, 0, st>>>(E, target, n, gE, loss);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- upload

// One CTA per probe, one thread per tile texel. dL/dE of an interior texel is
// its own loss gradient plus the atlas gradient of every tile texel that holds
// a copy of it; the filter's adjoint then scatters into the 3x3 neighbourhood.
__global__ void __launch_bounds__(64) k_upload_bwd(DevCascade C, DevParams P, const float4* H, const float4* gE,
                                                   const float4* gA, float4* gH) {
    __shared__ float4 h[36];
    __shared__ float gOut[36][3];
    __shared__ float gIn[36][4];
    const uint32_t p = blockIdx.x, t = threadIdx.x;
    if (t < 36) {
        h[t] = H[(size_t)p * 64u + interior_local(t)];
        float4 g = gE ? gE[(size_t)p * 36u + t] : make_float4(0.f, 0.f, 0.f, 0.f);
        gOut[t][0] = g.x;
        gOut[t][1] = g.y;
        gOut[t][2] = g.z;
        gIn[t][0] = gIn[t][1] = gIn[t][2] = gIn[t][3] = 0.0f;
    }
    __syncthreads();
    if (gA) {
        const uint32_t lx = t % TILE, ly = t / TILE;
        float4 g = gA[tile_texel(C, p, lx, ly)];
        sh_add3(gOut[gutter_source(lx, ly)], xyz(g));
    }
    __syncthreads();
    if (t < 36) {
        const int sx = (int)(t % OCT), sy = (int)(t / OCT);
        float4 c4 = h[t];
        float3 eC = xyz(c4);
        float lumaC = luma3(eC);
        float varRaw = c4.w - lumaC * lumaC;
        float varC = fmaxf(varRaw, 0.0f);
        float smW = 1.0f + P.filterSmooth * 6.0f;
        float kEff = 8.0f * smW * P.debugFilterKScale;
        float relEff = 0.0225f * smW * P.debugFilterRelScale;
        float epsF = 0.001f * P.debugFilterEpsScale;
        float inner = fmaxf(epsF, lumaC * lumaC * relEff);
        float denRaw = varC * kEff + inner;
        float den = fmaxf(denRaw, 1e-8f);
        float3 facc = mk(0.f, 0.f, 0.f);
        float fw = 0.0f, w[9], dl[9];
        uint32_t nb[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int jx = q % 3 - 1, jy = q / 3 - 1;
            const float gw = (jx == 0 && jy == 0) ? 1.0f : (jx == 0 || jy == 0) ? 0.6065306597126334f
                                                                                 : 0.36787944117144233f;
            int nx = min(max(sx + jx, 0), OCT - 1), ny = min(max(sy + jy, 0), OCT - 1);
            nb[q] = (uint32_t)(ny * OCT + nx);
            float3 en = xyz(h[nb[q]]);
            dl[q] = luma3(en) - lumaC;
            w[q] = gw * expf(dl[q] * dl[q] / den * -1.0f);
            facc = facc + en * w[q];
            fw += w[q];
        }
        const float fden = fmaxf(fw, 1e-4f);
        const float s = P.filterStrength;
        const float3 g = mk(gOut[t][0], gOut[t][1], gOut[t][2]);
        float3 gEC = g * (1.0f - s);
        const float3 gFilt = g * s;
        const float3 gFacc = gFilt * (1.0f / fden);
        const float gFw = fw > 1e-4f ? -dot3(gFilt, facc) / (fden * fden) : 0.0f;
        float gDen = 0.0f, gLumaC = 0.0f;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            float3 en = xyz(h[nb[q]]);
            float gW = dot3(gFacc, en) + gFw;
            float gq = -gW * w[q];                // d/d(dl^2 / den): w = gw exp(-q)
            float gDl = gq * 2.0f * dl[q] / den;
            gDen -= gq * dl[q] * dl[q] / (den * den);
            sh_add3(gIn[nb[q]], gFacc * w[q] + lumaw3(gDl));
            gLumaC -= gDl;
        }
        if (denRaw > 1e-8f) {
            float gVarC = gDen * kEff;
            if (lumaC * lumaC * relEff > epsF) gLumaC += gDen * 2.0f * lumaC * relEff;
            if (varRaw > 0.0f) {
                atomicAdd(&gIn[t][3], gVarC);
                gLumaC -= 2.0f * lumaC * gVarC;
            }
        }
        gEC = gEC + lumaw3(gLumaC);
        sh_add3(gIn[t], gEC);
    }
    __syncthreads();
    if (t < 36) {
        const size_t i = (size_t)p * 64u + interior_local(t);
        float4 o = gH[i];
        gH[i] = make_float4(o.x + gIn[t][0], o.y + gIn[t][1], o.z + gIn[t][2], o.w + gIn[t][3]);
    }
}

cudaError_t launch_upload_bwd(const DevCascade& C, const DevParams& P, const float4* H, const float4* gE,
                              const float4* gA, float4* gH, cudaStream_t st) {
    if (C.probeTotal == 0) return cudaSuccess;
    k_upload_bwd<<<C.probeTotal, 64, 0, st>>>(C, P, H, gE, gA, gH);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- blend

constexpr int BWD_CHUNK = 64;
constexpr int BWD_THREADS = 128;

struct BlendBwdSmem {
    float4 texDir[36];
    float4 rayDir[BWD_CHUNK];
    float wc[BWD_CHUNK][36];
    float4 fa[BWD_CHUNK];     // r, g, b, luma
    float4 cM[36];            // dL/d(meanRad) / wden, dL/d(curL) / wden
    float cM2[36];            // dL/d(curM2) / wden
};

// The 36 x n cosine-weight table of rays [c, c + n) and their radiance
// features, exactly as k_blend_upload forms them.
__device__ __forceinline__ void bwd_stage(BlendBwdSmem& S, const DevCascade& C, const DevParams& P, const float4* rays,
                                          uint32_t p, uint32_t c, uint32_t n, float cosPow, bool cosUnit) {
    const uint32_t N = C.rays;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        float4 r = rays[(size_t)p * N + c + k];
        S.fa[k] = make_float4(r.x, r.y, r.z, luma3(xyz(r)));
        float3 d = ray_dir(c + k, N, P.frameJitter);
        S.rayDir[k] = make_float4(d.x, d.y, d.z, 0.0f);
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < n * 36u; e += blockDim.x) {
        uint32_t k = e / 36u, j = e % 36u;
        float4 a = S.texDir[j], b = S.rayDir[k];
        float cd = fmaxf(a.x * b.x + a.y * b.y + a.z * b.z, 0.0f);
        S.wc[k][j] = cosUnit ? cd : powf(cd, cosPow);
    }
    __syncthreads();
}

// One CTA per probe. Pass 1 re-forms the texel moments (same order and
// operations as the forward); the temporal adjoint runs per texel; pass 2
// gives each ray sum_j wc[k][j] * (dMean_j + luma_w (dL_j + 2 l_k dM2_j)).
__global__ void __launch_bounds__(BWD_THREADS) k_blend_bwd(DevCascade C, DevParams P, const float4* rays,
                                                           const float4* Hprev, const float4* gH, float4* gHprev,
                                                           float4* gR) {
    __shared__ BlendBwdSmem S;
    const uint32_t p = blockIdx.x, tid = threadIdx.x, N = C.rays;
    const float cosPow = fmaxf(P.debugCosinePower, 1e-4f);
    const bool cosUnit = cosPow == 1.0f;
    if (tid < 36) {
        float u = (float(tid % OCT) + 0.5f) / 6.0f, v = (float(tid / OCT) + 0.5f) / 6.0f;
        float3 d = oct_decode(u, v);
        S.texDir[tid] = make_float4(d.x, d.y, d.z, 0.0f);
    }
    float sr = 0.f, sg = 0.f, sb = 0.f, sl = 0.f, sl2 = 0.f, ws = 0.f;
    float cr = 0.f, cg = 0.f, cb = 0.f, cl = 0.f, cl2 = 0.f, cws = 0.f;
    for (uint32_t c = 0; c < N; c += BWD_CHUNK) {
        const uint32_t n = min((uint32_t)BWD_CHUNK, N - c);
        __syncthreads();
        bwd_stage(S, C, P, rays, p, c, n, cosPow, cosUnit);
        if (tid < 36) {
            for (uint32_t k = 0; k < n; ++k) {  // the forward's compensated sums, same order
                float w = S.wc[k][tid];
                float4 a = S.fa[k];
                kahan_fma(sr, cr, w, a.x);
                kahan_fma(sg, cg, w, a.y);
                kahan_fma(sb, cb, w, a.z);
                kahan_fma(sl, cl, w, a.w);
                kahan_fma(sl2, cl2, w, a.w * a.w);
                kahan_fma(ws, cws, w, 1.0f);
            }
        }
    }
    if (tid < 64) {
        // non-interior history entries carry no gradient
        const uint32_t lx = tid % TILE, ly = tid / TILE;
        if (lx < BORDER || lx >= BORDER + OCT || ly < BORDER || ly >= BORDER + OCT)
            gHprev[(size_t)p * 64u + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (tid < 36) {
        const size_t ib = (size_t)p * 64u + interior_local(tid);
        const float wden = fmaxf(ws, 1e-4f);
        const float3 meanRad = mk(sr / wden, sg / wden, sb / wden);
        const float curL = sl / wden, curM2 = sl2 / wden;
        const float4 prev4 = Hprev[ib];
        const float3 prev = xyz(prev4);
        const float prevM2 = prev4.w;
        const float4 go = gH[ib];
        const float3 gBl = xyz(go);
        const float gM2 = go.w;
        float3 gMean = mk(0.f, 0.f, 0.f), gPrev = mk(0.f, 0.f, 0.f);
        float gCurL = 0.f, gCurM2 = 0.f, gPrevM2 = 0.f;
        const bool wasBlack = (prev.x + prev.y + prev.z) < 1e-6f;
        if (wasBlack) {  // h = 0: blended = meanRad, m2 = curM2
            gMean = gBl;
            gCurM2 = gM2;
        } else {
            const float prevL = luma3(prev);
            const float prevVarRaw = prevM2 - prevL * prevL, curVarRaw = curM2 - curL * curL;
            const float prevVar = fmaxf(prevVarRaw, 0.0f), curVar = fmaxf(curVarRaw, 0.0f);
            const float lumRef = fmaxf(fmaxf(curL, prevL), 0.0f);
            const float varFloor = P.debugTempVarEps + lumRef * lumRef * P.debugTempVarRel;
            const float sigma = sqrtf(prevVar + curVar + varFloor);
            const float delta = curL - prevL, absDelta = fabsf(delta);
            const float c0 = P.debugTempChangeSigma0, c1 = fmaxf(P.tempChangeSigma1, P.debugTempChangeSigma0 + 0.01f);
            const float s0 = sigma * c0, s1 = sigma * c1;
            const float cden = fmaxf(s1 - s0, 1e-6f);
            const float x = (absDelta - s0) / cden;
            const float changeW = clampf(x, 0.0f, 1.0f);
            const float Hh = P.hysteresis;
            const float rawNoiseH = Hh + (1.0f - Hh) * P.debugTempNoiseHBoost;
            const float rawChangeH = fmaxf(Hh - P.tempChangeHDrop, P.debugTempMinChangeH);
            const float rawHEff = mixf(rawNoiseH, rawChangeH, changeW);
            const float hc = clampf(rawHEff, 1e-6f, 1.0f);
            const float h = powf(hc, P.hysteresisExponent);
            const float bandIn = prevVar + varFloor;
            const float band = sqrtf(bandIn) * P.tempClampSigma;
            const float D = fmaxf(absDelta, 1e-6f);
            const float ratio = band / D;
            const float cs = fminf(1.0f, ratio);
            const float3 cand = prev + (meanRad - prev) * cs;
            // blended = cand (1 - h) + prev h;  m2 = curM2 (1 - h) + prevM2 h
            const float3 gCand = gBl * (1.0f - h);
            gPrev = gBl * h;
            gCurM2 = gM2 * (1.0f - h);
            gPrevM2 = gM2 * h;
            const float gh = dot3(gBl, prev - cand) + gM2 * (prevM2 - curM2);
            // cand = prev + (meanRad - prev) cs
            gMean = gCand * cs;
            gPrev = gPrev + gCand * (1.0f - cs);
            const float gcs = dot3(gCand, meanRad - prev);
            float gAbs = 0.f, gPrevVar = 0.f, gCurVar = 0.f, gVarFloor = 0.f;
            if (ratio < 1.0f) {
                const float gBand = gcs / D;
                if (absDelta > 1e-6f) gAbs -= gcs * ratio / D;
                if (bandIn > 0.0f) {
                    const float gIn = gBand * P.tempClampSigma * 0.5f / sqrtf(bandIn);
                    gPrevVar += gIn;
                    gVarFloor += gIn;
                }
            }
            // h = pow(clamp(raw), exponent), raw = mix(noiseH, changeH, changeW)
            if (rawHEff > 1e-6f && rawHEff < 1.0f) {
                const float gRaw = gh * P.hysteresisExponent * powf(hc, P.hysteresisExponent - 1.0f);
                const float gChange = gRaw * (rawChangeH - rawNoiseH);
                if (x > 0.0f && x < 1.0f) {
                    gAbs += gChange / cden;
                    float gs0 = -gChange / cden, gs1 = 0.f;
                    if (s1 - s0 > 1e-6f) {
                        const float gCden = -gChange * x / cden;
                        gs1 += gCden;
                        gs0 -= gCden;
                    }
                    const float gSigma = gs0 * c0 + gs1 * c1;
                    if (sigma > 0.0f) {
                        const float gV = gSigma * 0.5f / sigma;
                        gPrevVar += gV;
                        gCurVar += gV;
                        gVarFloor += gV;
                    }
                }
            }
            float gPrevL = 0.f;
            const float gLumRef = gVarFloor * 2.0f * lumRef * P.debugTempVarRel;
            if (lumRef > 0.0f) {
                if (curL >= prevL) gCurL += gLumRef;
                else gPrevL += gLumRef;
            }
            const float sgn = delta >= 0.0f ? 1.0f : -1.0f;
            gCurL += gAbs * sgn;
            gPrevL -= gAbs * sgn;
            if (curVarRaw > 0.0f) {
                gCurM2 += gCurVar;
                gCurL -= 2.0f * curL * gCurVar;
            }
            if (prevVarRaw > 0.0f) {
                gPrevM2 += gPrevVar;
                gPrevL -= 2.0f * prevL * gPrevVar;
            }
            gPrev = gPrev + lumaw3(gPrevL);
        }
        gHprev[ib] = make_float4(gPrev.x, gPrev.y, gPrev.z, gPrevM2);
        const float inv = 1.0f / wden;
        S.cM[tid] = make_float4(gMean.x * inv, gMean.y * inv, gMean.z * inv, gCurL * inv);
        S.cM2[tid] = gCurM2 * inv;
    }
    for (uint32_t c = 0; c < N; c += BWD_CHUNK) {
        const uint32_t n = min((uint32_t)BWD_CHUNK, N - c);
        __syncthreads();
        bwd_stage(S, C, P, rays, p, c, n, cosPow, cosUnit);
        for (uint32_t k = tid; k < n; k += blockDim.x) {
            const float l = S.fa[k].w;
            float3 g = mk(0.f, 0.f, 0.f);
            float gl = 0.f;
            for (uint32_t j = 0; j < 36; ++j) {
                const float w = S.wc[k][j];
                const float4 m = S.cM[j];
                g = g + mk(m.x, m.y, m.z) * w;
                gl = fmaf(w, m.w + 2.0f * l * S.cM2[j], gl);
            }
            g = g + lumaw3(gl);
            gR[(size_t)p * N + c + k] = make_float4(g.x, g.y, g.z, 0.0f);
        }
    }
}

cudaError_t launch_blend_bwd(const DevCascade& C, const DevParams& P, const float4* rays, const float4* Hprev,
                             const float4* gH, float4* gHprev, float4* gR, cudaStream_t st) {
    if (C.probeTotal == 0) return cudaSuccess;
    k_blend_bwd<<<C.probeTotal, BWD_THREADS, 0, st>>>(C, P, rays, Hprev, gH, gHprev, gR);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- shade

// The 32 texel taps of sample_atlas (8 cage probes x bilinear 2x2) with their
// normalised weights: sample = sum_i w_i * atlas[texel_i].
__device__ __forceinline__ void atlas_taps(const DevCascade& C, float3 P, float3 N, uint32_t* idx, float* wt) {
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
    // the footprint and weights of sample_atlas (tile-local, the same for all taps)
    const float2 ouv = oct_encode(normalize3(N));
    const float xl = fmaf(ouv.x, 6.0f, 0.5f), yl = fmaf(ouv.y, 6.0f, 0.5f);
    const float fx0 = floorf(xl), fy0 = floorf(yl), fx = xl - fx0, fy = yl - fy0;
    const uint32_t Wu = C.atlasW, off = (uint32_t)fy0 * Wu + (uint32_t)fx0;
    float wsum = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        float px = base[0] + float(dx), py = base[1] + float(dy), pz = base[2] + float(dz);
        float wx = dx ? frac[0] : 1.0f - frac[0];
        float wy = dy ? frac[1] : 1.0f - frac[1];
        float wz = dz ? frac[2] : 1.0f - frac[2];
        float w = wx * wy * wz + 1e-4f;
        const uint32_t t = ((uint32_t)pz * C.res[1] + (uint32_t)py) * 8u * Wu + (uint32_t)px * 8u + off;
        idx[4 * i] = t;
        idx[4 * i + 1] = t + 1u;
        idx[4 * i + 2] = t + Wu;
        idx[4 * i + 3] = t + Wu + 1u;
        wt[4 * i] = w * (1.0f - fx) * (1.0f - fy);
        wt[4 * i + 1] = w * fx * (1.0f - fy);
        wt[4 * i + 2] = w * (1.0f - fx) * fy;
        wt[4 * i + 3] = w * fx * fy;
        wsum += w;
    }
    const float inv = 1.0f / fmaxf(wsum, 1e-4f);
#pragma unroll
    for (int i = 0; i < 32; ++i) wt[i] *= inv;
}

constexpr int SHADE_BWD_THREADS = 256;

// One thread per ray. Parameter gradients gather per CTA in shared memory
// (FP32) and flush with one FP64 atomic per touched entry; atlas gradients go
// straight to global memory as float4 atomics.
__global__ void __launch_bounds__(SHADE_BWD_THREADS) k_shade_bwd(WaveCtx W, const float4* gR, double* gParam,
                                                                 float4* gA, uint32_t nParam, int useSmem) {
    extern __shared__ float sParam[];
    if (!*W.S.valid) return;
    const DevCascade& C = W.C;
    const DevParams& P = W.P;
    const uint32_t N = C.rays, mc = W.S.materialCount;
    if (useSmem) {
        for (uint32_t i = threadIdx.x; i < nParam; i += blockDim.x) sParam[i] = 0.0f;
        __syncthreads();
    }
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < C.probeTotal * N) {
        const uint32_t slot = g / N, k = g - slot * N;
        const uint4 hrec = C.hits[g];
        const float3 gr = xyz(gR[g]);
        if (hrec.x != 0xFFFFFFFFu && (gr.x != 0.f || gr.y != 0.f || gr.z != 0.f)) {
            const uint32_t tri = hrec.x, inst = hrec.y & 0x7FFFFFFFu;
            const float3 ro = probe_world_pos(C, slot);
            const float3 rd = ray_dir(k, N, P.frameJitter);
            const HitFrame fr = hit_frame(W, tri, inst, ro, rd, __uint_as_float(hrec.z), (int)(hrec.y >> 31));
            const uint32_t m = __ldg(W.S.triMaterial + tri);
            const float* M = W.S.materials + (size_t)m * 28u;
            const float3 baseColor = mk(__ldg(M), __ldg(M + 1), __ldg(M + 2));
            const float metal = __ldg(M + 4), transm = __ldg(M + 5);
            const float kdScale = P.debugAlbedoScale * (1.0f - metal) * (1.0f - transm);
            const float3 kdr = baseColor * kdScale;
            const float3 kd = mk(clampf(kdr.x, 0.f, 0.95f), clampf(kdr.y, 0.f, 0.95f), clampf(kdr.z, 0.f, 0.95f));
            float3 gkd = mk(0.f, 0.f, 0.f);
            // emissive: radiance += emissive * debugEmissiveScale
            const float3 gEm = gr * P.debugEmissiveScale;
            // unblocked NEE lights: term = kd (.) X, linear in the light's colour
            const uint4 v = C.vis[g];
            unsigned long long ok = (unsigned long long)v.z | ((unsigned long long)v.w << 32);
            while (ok) {
                const uint32_t li = (uint32_t)(__ffsll((long long)ok) - 1);
                ok &= ok - 1ull;
                const LightEval e = light_eval(W, li, fr.hitPos, fr.ng);
                const float3 X = light_term(W, e, mk(1.f, 1.f, 1.f));
                const float3 term = mul3(X, kd);
                const float gl = dot3(gr, term);
                gkd = gkd + mul3(gr, X);
                if (useSmem) atomicAdd(&sParam[6u * mc + li], gl);
                else atomicAdd(&gParam[6u * mc + li], (double)gl);
            }
            // bounce = sample (.) kd / pi, scaled by roll = C / max(C, luma(bounce))
            uint32_t idx[32];
            float wt[32];
            atlas_taps(C, fr.hitPos, fr.ng, idx, wt);
            float3 smp = mk(0.f, 0.f, 0.f);
#pragma unroll
            for (int i = 0; i < 32; ++i) smp = smp + xyz(half4_to_float4(__ldg(C.atlasPrev + idx[i]))) * wt[i];
            const float3 bounce = mul3(smp, kd) * (1.0f / PI_F);
            const float bl = luma3(bounce);
            const float Cc = P.radianceClamp;
            const float rden = fmaxf(fmaxf(Cc, bl), 1e-6f);
            float3 gB;
            if (bl > Cc && bl > 1e-6f) {
                const float k1 = Cc * P.debugBounceScale / rden;
                gB = gr * k1 - lumaw3(dot3(gr, bounce) * k1 / rden);
            } else {
                gB = gr * (Cc / rden * P.debugBounceScale);
            }
            const float3 gS = mul3(gB, kd) * (1.0f / PI_F);
            gkd = gkd + mul3(gB, smp) * (1.0f / PI_F);
#pragma unroll 4
            for (int i = 0; i < 32; ++i) {
                const float3 a = gS * wt[i];
                atomicAdd(gA + idx[i], make_float4(a.x, a.y, a.z, 0.0f));
            }
            const float3 gBase = mk(kdr.x > 0.f && kdr.x < 0.95f ? gkd.x * kdScale : 0.f,
                                    kdr.y > 0.f && kdr.y < 0.95f ? gkd.y * kdScale : 0.f,
                                    kdr.z > 0.f && kdr.z < 0.95f ? gkd.z * kdScale : 0.f);
            if (useSmem) {
                sh_add3(sParam + 3u * m, gBase);
                sh_add3(sParam + 3u * (mc + m), gEm);
            } else {
                for (int c = 0; c < 3; ++c) {
                    atomicAdd(&gParam[3u * m + c], (double)(&gBase.x)[c]);
                    atomicAdd(&gParam[3u * (mc + m) + c], (double)(&gEm.x)[c]);
                }
            }
        }
    }
    if (useSmem) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nParam; i += blockDim.x)
            if (sParam[i] != 0.0f) atomicAdd(&gParam[i], (double)sParam[i]);
    }
}

cudaError_t launch_shade_bwd(const DevScene& S, const DevCascade& C, const DevParams& P, const float4* gR,
                             double* gParam, float4* gA, cudaStream_t st) {
    const uint32_t rays = C.probeTotal * C.rays;
    if (rays == 0) return cudaSuccess;
    WaveCtx W{};
    W.S = S;
    W.C = C;
    W.P = P;
    W.slotCount = C.probeTotal;
    const uint32_t nParam = 6u * S.materialCount + S.lightCount;
    const size_t smem = (size_t)nParam * sizeof(float);
    const int useSmem = smem <= 32u * 1024u ? 1 : 0;
    k_shade_bwd<<<(rays + SHADE_BWD_THREADS - 1) / SHADE_BWD_THREADS, SHADE_BWD_THREADS, useSmem ? smem : 0, st>>>(
        W, gR, gParam, gA, nParam, useSmem);
    note_launch();
    return cudaGetLastError();
}

}  // namespace sb
