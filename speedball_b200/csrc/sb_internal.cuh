// sb_internal.cuh — device-side structures and helpers shared by the CUDA
// translation units of libspeedball_cuda.so (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include "../../include/speedball_cuda.h"

namespace sb {

// Device error word bits (latched; read back by sb_synchronize).
enum : uint32_t {
    ERR_LAYOUT = 1u,      // threaded-layout / index-range violation
    ERR_WATCHDOG = 2u,    // a bounded loop ran out of iterations
    ERR_NAN_KEY = 4u,     // NaN TLAS build key (instance AABB)
    ERR_CAPACITY = 8u,    // a device-side capacity was exceeded
};

constexpr uint32_t INTERIOR = 0xFFFFFFFFu;
constexpr float RAY_EPS = 1e-3f;
constexpr float T_MAX = 1e30f;
constexpr float PI_F = 3.141592653589793f;
constexpr int OCT = 6, TILE = 8, BORDER = 1;
constexpr uint32_t LIGHT_DATA = 64u * 17u;  // records before the C0 cell lists

// Child-pair nodes (derived, 64 bytes per interior node, indexed like the
// reference nodes): q0 = child0 (minx, maxx, miny, maxy), q1 = child1 (same),
// q2 = (child0 minz, maxz, child1 minz, maxz), q3 = (entry0, entry1, 0, 0).
// An entry names what a traversal does next with that child:
//   top byte != 0           BLAS leaf: the reference payload (cnt << 24) | triOffset
//   PE_BLAS | node          BLAS interior node (node < 2^23)
//   PE_TLEAF | cnt<<12 | s  TLAS leaf: cnt instance slots from s (s < 4096, cnt < 1024)
//   node                    TLAS interior node (node < 2^22)
//   PE_NONE                 nothing to visit (an empty leaf)
constexpr uint32_t PE_NONE = 0xFFFFFFFFu;
constexpr uint32_t PE_BLAS = 0x00800000u;
constexpr uint32_t PE_TLEAF = 0x00400000u;
constexpr uint32_t PE_BLAS_MAX_NODES = 1u << 23;
constexpr uint32_t PE_TLAS_MAX_SLOTS = 4096u;
constexpr uint32_t DEPTH_UNKNOWN = 0xFFFFFFFFu;

// Entries of the per-thread traversal stack (child-pair and scene-BVH walks).
#ifndef SB_STACK
#define SB_STACK 40
// default per-ray node-step limits of the walks (sb_set_walk_step_limit)
#define SB_WALK_STEPS_DEFAULT (1u << 26)
#define SB_WALK_STEPS_REF_DEFAULT (1u << 28)
#endif

// Per-triangle accept bits packed in the w lane of the first float4 of a
// pre-gathered triangle (materialSideAccepts / materialAlphaAccepts /
// traversal flags, spectral_traverse.js:193-222 with no map bound).
enum : uint32_t {
    TB_SIDE_MASK = 3u,      // 0 front, 1 back, 2 double
    TB_CLOSEST_OK = 4u,     // closest-hit alpha acceptance
    TB_SHADOW_OK = 8u,      // any-hit: shadow-block flag and alpha acceptance
};

// Scene as the kernels see it. Reference layouts are kept for refit and
// read-back; the kernels traverse the derived layouts.
struct DevScene {
    const uint4* nodes;        // 2 x uint4 per BLAS node: bmin.xyz bmax.x | bmax.yz miss payload
    const float4* tris;        // 3 x float4 per triangle: (p0, bits) (e1, -) (e2, -)
    const uint32_t* triMaterial;
    const float* materials;    // uber records (28 floats)
    const float4* inst;        // 4 x float4 per instance slot: 3 inverse rows, (root, end, dSign, active)
    const uint4* tlas;         // 2 x uint4 per TLAS node, same encoding as BLAS nodes, payload (cnt<<24)|off
    const float* lights;       // 64 x 17 records (+ C0 cell lists)
    const float4* lightGates;  // the records' gate fields, 3 x float4 per light
    const uint32_t* triIndex;  // reference triangle indices (final-hit refinement)
    const float* vertexData;   // reference vertices, 8 floats each
    const uint4* pairs;        // 4 x uint4 per interior BLAS node: both children's boxes + entries
    const uint4* tlasPairs;    // the same for interior TLAS nodes
    const uint32_t* depth;     // [0] deepest BLAS node, [1] deepest TLAS node (NONE: pairs unusable)
    // scene BVH (sb_flat.h): world-space tree over (triangle, slot) items;
    // slots marked in slotSkip moved or deformed since its build and are
    // walked through their own BLAS instead (dynList)
    const uint4* flatNodes;    // binary child pairs (any hit; closest hit when wideNodes is null)
    const uint2* flatItems;
    const uint4* wideNodes;    // the same items as 8-wide nodes with 8-bit boxes (closest hit), or null
    const uint2* wideItems;
    const uint8_t* slotSkip;
    const uint32_t* dynList;
    const float* slotBounds;   // world AABB per slot (the TLAS leaf bounds), or null
    uint32_t flatRoot, dynCount;
    uint32_t wideNodeCount;    // nodes of the 8-wide tree (0 when it is not built)
    uint32_t wideDepth;        // its depth (levels below the root)
    int32_t flatOn;
    uint32_t nodeCount, triCount, instCount, tlasNodeCount, materialCount;
    uint32_t lightCount;
    int32_t clustered;
    const uint32_t* valid;     // nonzero when the last pack validated the layout
    // per-ray step limits of the walks (node visits; a walk that reaches its
    // limit latches ERR_WATCHDOG and ends): iterCap for the scene-BVH walks,
    // iterCapRef for the reference's TLAS + BLAS walks
    uint32_t iterCap, iterCapRef;
};

// One cascade solve as the kernels see it.
struct DevCascade {
    float gridMin[3], gridSize[3];
    uint32_t res[3];
    uint32_t rays;
    float maxDist, cellMin;
    uint32_t probeTotal, atlasW, atlasH;
    uint32_t probeOffset, updatedCount;
    // cascade 0's grid, for the clustered cell lookup
    float g0Min[3], g0Size[3];
    uint32_t g0Res[3];
    float4* rayData;           // updatedCount*rays
    uint4* hits;               // 16-byte hit records: tri, inst | facing << 31, t, packed uv
    uint4* vis;                // NEE masks: tested lights (lo, hi), unblocked lights (lo, hi)
    float4* irr;               // history, probeTotal*64
    float2* depth;             // history
    const uint2* atlasPrev;    // RGBA16F texels as 4 halves (the previous upload)
    uint2* atlas;              // RGBA16F output
    uint2* depthAtlas;
    float4* eOut;              // optional: FP32 upload output of the 36 interior texels per probe (adjoint tape)
    const uint32_t* issueOrder;  // optional (full updates from slot 0): direction-major issue visits the
                                 // probes in this order, 32 per compact 4 x 4 x 2 tile
    // optional (sortKey 3, with issueOrder): the closest-hit stage hands out its 32-ray batches
    // in batchOrder (costliest of the previous solve first) and records each batch's cycles in
    // batchCost; the shadow stage's first idle CTA writes the next solve's order to batchOrderOut
    const uint32_t* batchOrder;
    uint32_t* batchCost;
    uint32_t* batchOrderOut;
    // giEmitter records (type 3) and this cascade's emitter visibility history,
    // probeTotal x EMITTER_CAP (gi_probes.js:1873, 2216-2310)
    const float* lights;
    uint32_t emitterBase, emitterCount;
    float* emitterVis;
    // reflection lobes (tier 0 off, 1 rough, 2 high, 3 ultra; gi_probes.js:60-75):
    // rough history probeTotal*64 and its RGBA16F atlas in the irradiance layout;
    // glossy numerator / support per glossy texel (probeTotal*glossyTile^2) and
    // the glossy atlas, tile of probe p at (p % glossyTilesX, p / glossyTilesX)
    uint32_t reflect;
    float4* roughSpec;
    uint2* roughAtlas;
    float4* glossyNum;
    float* glossyDen;
    uint2* glossyAtlas;
    uint32_t glossyOct, glossyTile, glossyInterval, glossyPhase, glossyTilesX, glossyAtlasW;
};
constexpr uint32_t EMITTER_CAP = 16;          // GI_EMITTER_INJECT_CAP, gi_probes.js:133
constexpr float EMITTER_VIS_RETENTION = 0.8f;  // GI_EMITTER_VIS_RETENTION, gi_probes.js:134
constexpr float ROUGH_UNSHADED_T_BIAS = 2.0f;  // gi_probes.js:94

struct DevParams {
    float frameJitter, emitterVisSeed;
    float hysteresis, hysteresisExponent;
    float depthSharpness, radianceClamp, classifyStrength;
    float filterStrength, filterSmooth;
    float tempChangeSigma1, tempChangeHDrop, tempClampSigma;
    float nirGate, nirGain;
    float skyIntensity;
    float skySH[27];
    float debugTraceBiasScale, debugRayEpsScale, debugDirectScale, debugEmissiveScale;
    float debugAlbedoScale, debugBounceScale, debugCosinePower;
    float debugTempNoiseHBoost, debugTempChangeSigma0, debugTempMinChangeH;
    float debugTempVarEps, debugTempVarRel, debugDepthHistoryScale;
    float debugFilterKScale, debugFilterRelScale, debugFilterEpsScale;
    float reflectionSkyFallback, skyConfigured;
};
static_assert(sizeof(DevParams) == sizeof(sb_params), "DevParams mirrors sb_params");

// One solve of the trace wavefront as its kernels see it.
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
    uint32_t smemWide;             // top 8-wide nodes staged in shared memory by the closest-hit stage
    uint32_t sstk;                 // closest-hit walk stack entries per thread in shared memory (0: local)
};

// Several solves (scenes, cascades) through one launch of each stage: a
// shared ray index space in which item i owns [rayBase, rayBase + rays), with
// rayBase a multiple of 32 so a warp's 32 rays never straddle two items, and a
// shared shadow-job queue whose jobs carry the global ray index. The blend
// grid is split the same way (blendBase / blendBlocks CTAs per item). Passed
// by value as a __grid_constant__ kernel parameter and indexed in place.
constexpr uint32_t SB_BATCH_MAX = 16;
struct BatchItem {
    WaveCtx W;                     // W.work / W.jobs / W.jobCap are the batch's shared ones
    uint32_t rayBase, rays;
    uint32_t blendBase, blendBlocks;
};
struct BatchArgs {
    BatchItem it[SB_BATCH_MAX];
    uint32_t n;
    uint32_t totalRays;            // padded ray index space
    uint32_t blendBlocks;
    uint32_t* work;
    unsigned long long* counters;  // one set for the whole batch, or null
};
static_assert(sizeof(BatchArgs) <= 32000, "BatchArgs must fit the kernel parameter space");

__device__ __forceinline__ uint32_t batch_item(const BatchArgs& B, uint32_t g) {
    uint32_t i = 0;
#pragma unroll 1
    while (i + 1 < B.n && g >= B.it[i + 1].rayBase) ++i;
    return i;
}

__device__ __forceinline__ void latch(uint32_t* err, uint32_t bit) {
    if (err) atomicOr(err, bit);
}

// JS Math.min / Math.max on floats: NaN-propagating, -0 < +0 (the interior
// unions of gi_refit.js use them).
__device__ __forceinline__ float js_min(float a, float b) {
    if (a != a || b != b) return __int_as_float(0x7fc00000);
    if (a == b) return signbit(a) ? a : b;
    return a < b ? a : b;
}
__device__ __forceinline__ float js_max(float a, float b) {
    if (a != a || b != b) return __int_as_float(0x7fc00000);
    if (a == b) return signbit(a) ? b : a;
    return a > b ? a : b;
}

}  // namespace sb
