/*
 * speedball_cuda.h — C ABI of the B200-native DDGI probe update.
 *
 * One context (sb_ctx) is one probe field over one resident scene on one GPU.
 * The host (the reference's JavaScript facade through an N-API addon, or the
 * Python mirror in speedball_b200/) keeps the scene build and the per-tick
 * scheduling; everything the reference submits through renderer.computeAsync
 * (gi_probes.js:3236, 3812, 3836) and the CPU refit / TLAS lanes
 * (gi_refit.js, spectral_scene.js:973-1003, 1402-1514, 1831-1927) run here
 * as CUDA kernels for sm_100a.
 *
 * Conventions
 *  - Plain pointers and sizes only. Host arrays are owned by the caller and
 *    copied; device memory is owned by the library.
 *  - Every call returns sb_status. No exception or abort crosses the ABI.
 *    sb_last_error() returns a message for the last non-OK status.
 *  - Work is enqueued on the context's stream (sb_set_stream). Calls that
 *    enqueue device work do not block; device-side faults found by the
 *    kernels' own checks (layout violations, traversal watchdogs) are latched
 *    in a device error word and returned by the next sb_synchronize().
 *  - A context is not thread-safe: one host thread per context, mirroring the
 *    reference's single-threaded tick with its inFlight guard
 *    (gi_probes.js:3141, 3473).
 *  - Buffers use the reference's wire layouts (spectral_scene.js:35-55,
 *    724-733, 1188-1240, 1339-1366); the library derives its own B200
 *    layouts (pre-gathered triangles, compact TLAS, instance rows) on device.
 */
#ifndef SPEEDBALL_CUDA_H
#define SPEEDBALL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB_ABI_VERSION 3u

/* Geometry of the reference's layouts (spectral_scene.js:35-55, gi_probes.js:53-56). */
#define SB_NODE_STRIDE_U32 8u   /* bvhNodes: 6 f32 bounds + miss + payload        */
#define SB_MAT_STRIDE 28u       /* materials / instance records (floats)           */
#define SB_TLAS_STRIDE_F32 12u  /* TLAS nodes in the materials tail (floats)       */
#define SB_LIGHT_STRIDE 17u     /* light records (floats)                          */
#define SB_VERTEX_STRIDE 8u     /* vertexData: pos(3) normal(3) uv(2)              */
#define SB_OCT_RES 6u           /* interior octahedral texels per axis             */
#define SB_TILE 8u              /* tile incl. 1-texel gutter                       */
#define SB_MAX_LIGHTS 64u       /* gi_probes.js:132                                */
#define SB_LIGHTS_PER_CELL 16u  /* gi_probes.js:135                                */
#define SB_MAX_CASCADES 4u

typedef enum sb_status {
    SB_OK = 0,
    SB_ERR_INVALID_ARG = 1,        /* bad pointer, size or range                     */
    SB_ERR_LAYOUT_VIOLATION = 2,   /* threaded-layout invariant broken: the caller
                                      must fall back to a full rebuild, as the
                                      reference does when refit returns false
                                      (gi_refit.js:30-33, gi_probes.js:4170, 4220) */
    SB_ERR_OOM = 3,
    SB_ERR_CUDA = 4,
    SB_ERR_DEVICE_WATCHDOG = 5,    /* a bounded device loop hit its iteration cap    */
    SB_ERR_UNSUPPORTED = 6,        /* a feature outside this library's scope         */
    SB_ERR_NO_DEVICE = 7,
    SB_ERR_NOT_READY = 8           /* call order: e.g. solve before scene upload     */
} sb_status;

typedef struct sb_ctx sb_ctx;

/* ---------------------------------------------------------------- lifetime */

typedef struct sb_device_opts {
    int32_t device;        /* CUDA ordinal                                         */
    uint32_t flags;        /* SB_CTX_* below                                       */
} sb_device_opts;

#define SB_CTX_RECORD_HITS 1u  /* accepted, no effect: the 16-byte hit records and
                                  visibility masks of the last solve are always kept
                                  (the shade stage and sb_backward read them)        */

/* createProbeField (gi_probes.js:945) minus the renderer: allocates the context. */
sb_status sb_create(const sb_device_opts* opts, sb_ctx** out);
/* dispose() (install.js:488-502): frees every device allocation. NULL is a no-op. */
void sb_destroy(sb_ctx* ctx);
const char* sb_last_error(const sb_ctx* ctx);
uint32_t sb_abi_version(void);
/* Attach a caller stream (a cudaStream_t passed as void*); NULL = library stream. */
sb_status sb_set_stream(sb_ctx* ctx, void* cuda_stream);
/* Wait for the context's stream and return the latched device error, if any. */
sb_status sb_synchronize(sb_ctx* ctx);
/* Per-ray node-step limit of every traversal walk (0 = the defaults: 2^26
 * steps on the scene BVH, 2^28 on the reference's TLAS + BLAS walk, and never
 * more BLAS steps than the pool has nodes). A walk that reaches the limit
 * ends, and the next sb_synchronize returns SB_ERR_DEVICE_WATCHDOG. Validated
 * layouts always end well inside the defaults (the reference's walks have no
 * such limit: its miss links only move forward, spectral_traverse.js:361,
 * 445); a small limit is how the watchdog path is exercised from the host. */
sb_status sb_set_walk_step_limit(sb_ctx* ctx, uint32_t steps);
/* Page-locked host staging memory for the per-frame uploads (vertex gathers,
 * matrices) and read-backs, so copies run at full PCIe / C2C rate. The JS addon
 * wraps such blocks as external ArrayBuffers. */
sb_status sb_host_alloc(size_t bytes, void** out);
void sb_host_free(void* p);

/* ------------------------------------------------------------------ scene */

/* The typed arrays buildSpectralScene returns (spectral_scene.js:2011-2033).
 * materials = [uberCount*28 | instCount*28 instance records | tlasNodeCount*12]. */
typedef struct sb_scene_view {
    const uint32_t* bvhNodes;   uint32_t nodeCount;
    const uint32_t* triIndex;   uint32_t triCount;
    const float* vertexData;    uint32_t vertexCount;
    const uint32_t* triMaterial;
    const float* materials;     uint32_t materialsLen;   /* floats */
    uint32_t materialCount;     /* uber records                                  */
    uint32_t instBase;          /* float index of instance 0 (= materialCount*28) */
    uint32_t instCount;
    uint32_t tlasBase;          /* float index of TLAS node 0                    */
    uint32_t tlasNodeCount;
} sb_scene_view;

sb_status sb_upload_scene(sb_ctx* ctx, const sb_scene_view* scene);

typedef enum sb_buffer {
    SB_BUF_BVH_NODES = 0,    /* u32 units            */
    SB_BUF_TRI_INDEX = 1,    /* u32 units            */
    SB_BUF_VERTEX_DATA = 2,  /* f32 units            */
    SB_BUF_TRI_MATERIAL = 3, /* u32 units            */
    SB_BUF_MATERIALS = 4,    /* f32 units (incl. instance + TLAS tail) */
    SB_BUF_LIGHTS = 5,       /* f32 units            */
    SB_BUF_IRRADIANCE_HISTORY = 6, /* f32, 4 per texel, probeTotal*64 texels (per cascade) */
    SB_BUF_DEPTH_HISTORY = 7,      /* f32, 2 per texel                                   */
    SB_BUF_IRRADIANCE_ATLAS = 8,   /* u16 binary16 RGBA, atlasW*atlasH*4                 */
    SB_BUF_DEPTH_ATLAS = 9,        /* u16 binary16 RGBA                                  */
    SB_BUF_RAY_DATA = 10,          /* f32, 4 per ray: rgb + hitT (-1 = miss)             */
    SB_BUF_HIT_RECORDS = 11,       /* u32, 4 per ray: tri, inst, t bits, packed uv        */
    SB_BUF_VISIBILITY = 12,        /* u32, 4 per ray: lights shadow-tested (lo, hi) and
                                      left unblocked (lo, hi), bit = light index 0..63   */
    SB_BUF_TLAS_ORDER = 13,        /* u32, slot -> source instance                       */
    SB_BUF_INSTANCE_BOUNDS = 14,   /* f32, 6 per slot (liveInstanceBounds)               */
    SB_BUF_RECORD_E = 15,          /* f32, 4 per interior texel (rgb, 1), probeTotal*36:
                                      the FP32 upload output of the last solve of the
                                      last sb_forward_record (read-only)                 */
    SB_BUF_EMITTER_VIS = 16,       /* f32, 16 per probe: giEmitter visibility history
                                      (per cascade, read-only)                          */
    SB_BUF_ROUGH_SPECULAR = 17,    /* f32, 4 per texel, probeTotal*64: the rough
                                      reflection history (rgb, coverage); reflection
                                      tiers rough/high/ultra                             */
    SB_BUF_ROUGH_ATLAS = 18,       /* u16 binary16 RGBA, atlasW*atlasH*4                 */
    SB_BUF_GLOSSY_SPECULAR = 19,   /* f32, 4 per glossy texel, probeTotal*glossyTile^2:
                                      per-ray-mean numerator (rgb, coverage); tiers
                                      high/ultra                                         */
    SB_BUF_GLOSSY_WEIGHT = 20,     /* f32, 1 per glossy texel: per-ray-mean support      */
    SB_BUF_GLOSSY_ATLAS = 21       /* u16 binary16 RGBA, glossyAtlasW*glossyAtlasH*4     */
} sb_buffer;

/* Ranged host->device write into a reference buffer (the copySceneStorageRanges /
 * markStorageDirty seam, gi_probes.js:1543-1561, 4239-4251). Derived layouts are
 * refreshed before the next solve. For history buffers `cascade` selects the
 * cascade through the high byte of `which` (which | cascade << 8). */
sb_status sb_upload_range(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count,
                          const void* src);
/* Device->host read of any buffer above (the _debugRead seam, gi_probes.js:4830-4841).
 * Synchronous: the copy is queued behind the context's work and waited for. */
sb_status sb_read_buffer(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count,
                         void* dst);
/* The same read, only queued on the context's stream (the reference's read is
 * asynchronous too: _debugRead resolves a mapAsync). `dst` is valid after the
 * next sb_synchronize; page-locked memory (sb_host_alloc) lets the copy run
 * without a host round trip between several reads. */
sb_status sb_read_buffer_async(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count,
                               void* dst);

/* ------------------------------------------------------------------ lights */

/* Light records of stride 17 (collectLights, spectral_scene.js:724-813), already
 * selected into the fixed arena by the host (fillLegacyLightArena /
 * fillGiLightArena, gi_probes.js:4297-4349). clustered != 0 builds the C0 cell
 * lists on device (lightGridKernel, gi_probes.js:1888-1938) from cascade 0's grid.
 * Records [emitterBase, emitterBase + emitterCount) are giEmitter spheres (type
 * 3: centre [1..3], surface radiance [7..9], radius [14], projected area A/4
 * [15]; collectEmitterRecords, spectral_scene.js:815-888), at most 16: every
 * sb_solve then runs emitterVisKernel (a shadow ray per updated probe and
 * emitter into a visibility history of retention 0.8, gi_probes.js:2216-2260)
 * and the blend adds each emitter as virtual rays (2262-2310). NEE skips them.
 * Batched solves and the adjoint return SB_ERR_UNSUPPORTED while emitters are
 * uploaded. */
sb_status sb_upload_lights(sb_ctx* ctx, const float* records, uint32_t count,
                           uint32_t emitterBase, uint32_t emitterCount, int32_t clustered);

/* ----------------------------------------------------------- probe field */

/* Per-cascade uniforms (makeCascadeU, gi_probes.js:1010-1024; rebuild 3341-3367). */
typedef struct sb_grid {
    float gridMin[3];
    float gridSize[3];
    uint32_t res[3];          /* probes per axis, 2..32                            */
    uint32_t raysPerProbe;    /* 32..256, multiple of 16 (gi_probes.js:988-992)    */
    float maxDist;            /* |gridSize| (gi_probes.js:3151)                    */
    float cellMin;            /* max(1e-4, min cell edge) (gi_probes.js:3364)      */
} sb_grid;

/* Shared compute uniforms U (gi_probes.js:1198-1255). */
typedef struct sb_params {
    float frameJitter, emitterVisSeed;
    float hysteresis, hysteresisExponent;
    float depthSharpness, radianceClamp, classifyStrength;
    float filterStrength, filterSmooth;
    float tempChangeSigma1, tempChangeHDrop, tempClampSigma;
    float nirGate, nirGain;
    float skyIntensity;
    float skySH[27];          /* 9 coefficients x RGB, THREE.SphericalHarmonics3 order */
    float debugTraceBiasScale, debugRayEpsScale, debugDirectScale, debugEmissiveScale;
    float debugAlbedoScale, debugBounceScale, debugCosinePower;
    float debugTempNoiseHBoost, debugTempChangeSigma0, debugTempMinChangeH;
    float debugTempVarEps, debugTempVarRel, debugDepthHistoryScale;
    float debugFilterKScale, debugFilterRelScale, debugFilterEpsScale;
    float reflectionSkyFallback; /* 1: a true miss feeds the reflection lobes with the
                                    sky (setReflectionSkyFallback, gi_probes.js:1320-1324) */
    float skyConfigured;         /* 1 once a sky has been given (gi_probes.js:1316)      */
} sb_params;

/* The reference's defaults (hysteresis = gated 0.60, gi_probes.js:146-149). */
void sb_params_defaults(sb_params* p);

/* (Re)configure a cascade: allocates ray scratch, histories and both RGBA16F
 * atlases, cleared (clearAtlasKernel, gi_probes.js:2690-2707). A same-dimension
 * reconfigure keeps the live history, as the reference's `reuse` does
 * (gi_probes.js:3124-3197). */
sb_status sb_configure_cascade(sb_ctx* ctx, uint32_t cascade, const sb_grid* grid);
sb_status sb_set_params(sb_ctx* ctx, const sb_params* params);

/* Reflection lobes, the reference's structural tier (reflectionQuality,
 * REFLECTION_QUALITY_TIERS and resolveReflectionQuality, gi_probes.js:60-75):
 *   SB_REFLECT_OFF   no lobe (the default);
 *   SB_REFLECT_ROUGH the blend also accumulates a power-8 lobe into a rough
 *                    specular history and atlas in the irradiance tile layout,
 *                    and hits on surfaces with no diffuse energy and no
 *                    emission are stored as hitT = -(t + 2) (gi_probes.js:
 *                    2055-2062, 2358-2404, 2505-2522, 2838-2843);
 *   SB_REFLECT_HIGH  rough + a power-64 glossy lobe on 8x8 octahedral tiles
 *                    (10x10 with the gutter), half of each tile's texels per
 *                    solve (glossyKernel, 2538-2686);
 *   SB_REFLECT_ULTRA rough + the glossy lobe on 16x16 tiles, every texel every
 *                    solve.
 * Applies to every configured cascade and to later configures: reallocates and
 * clears the reflection histories and atlases and resets the glossy phase.
 * Batched solves and the adjoint return SB_ERR_UNSUPPORTED while a tier other
 * than off is set. */
typedef enum sb_reflect_tier {
    SB_REFLECT_OFF = 0, SB_REFLECT_ROUGH = 1, SB_REFLECT_HIGH = 2, SB_REFLECT_ULTRA = 3
} sb_reflect_tier;
sb_status sb_set_reflection_quality(sb_ctx* ctx, uint32_t tier);

/* A cascade's reflection layout. The glossy atlas packs probe p's tile at
 * column p % glossyTilesX, row p / glossyTilesX (glossyTilesX = ceil(sqrt(
 * probeTotal)), gi_probes.js:3103-3110); glossyPhase is the texel phase the
 * next solve of the cascade resolves (texels with local % glossyInterval ==
 * phase; 2561-2567, 3832-3835). */
typedef struct sb_reflection_layout {
    uint32_t tier;
    uint32_t glossyOct, glossyTile, glossyInterval;
    uint32_t glossyTilesX, glossyTilesY, glossyAtlasW, glossyAtlasH;
    uint32_t glossyPhase;
} sb_reflection_layout;
sb_status sb_get_reflection_layout(sb_ctx* ctx, uint32_t cascade, sb_reflection_layout* out);

/* One solve of one cascade: trace -> NEE/bounce shade -> blend -> upload for
 * probes (probeOffset + slot) mod probeTotal, slot < updatedCount (the
 * solveKernels pass, gi_probes.js:3815-3836). Enqueue only. */
sb_status sb_solve(sb_ctx* ctx, uint32_t cascade, uint32_t probeOffset, uint32_t updatedCount);

/* The batched form: solves of several contexts (scenes) and cascades through
 * one launch per stage: one persistent closest-hit launch over a shared ray
 * queue, one job-emission launch, one persistent shadow launch over a shared
 * job queue, one shade launch and one blend/upload launch for all items.
 * At most 16 items, all on one device, no (context, cascade) twice; the batch
 * runs on items[0].ctx's stream (which also owns the queues), ordered after
 * the other contexts' pending work and before their later work. Each item's
 * results equal those of sb_solve with the same arguments. Enqueue only;
 * device errors latch in each item's own context. */
typedef struct sb_solve_item {
    sb_ctx* ctx;
    uint32_t cascade, probeOffset, updatedCount;
} sb_solve_item;
sb_status sb_solve_batch(const sb_solve_item* items, uint32_t count);

/* Arbitrary-ray queries through the same two-level traversal (the reference's
 * traverseClosest / traverseAny, spectral_traverse.js:441-474, 539-569), host
 * arrays in and out; synchronous. ro/rd: 3 floats per ray. tri = -1 on a miss. */
sb_status sb_raycast(sb_ctx* ctx, const float* ro, const float* rd, uint32_t n, float* tOut,
                     int32_t* triOut, int32_t* instOut);
sb_status sb_occluded(sb_ctx* ctx, const float* ro, const float* rd, const float* maxDist,
                      uint32_t n, uint8_t* blockedOut);
/* The same two queries on DEVICE arrays (3 floats per ray; t, tri, inst per
 * ray; one byte per ray), enqueued on the context's stream with no copy and
 * no synchronisation: the traversal reused by a GPU path tracer, as the
 * reference's spectral kernel reuses traverseClosest / traverseAny
 * (spectral_kernel.js:288, 451). Results equal sb_raycast / sb_occluded. */
sb_status sb_raycast_device(sb_ctx* ctx, const float* ro, const float* rd, uint32_t n, float* tOut,
                            int32_t* triOut, int32_t* instOut);
sb_status sb_occluded_device(sb_ctx* ctx, const float* ro, const float* rd, const float* maxDist,
                             uint32_t n, uint8_t* blockedOut);

/* The FP32 probe rays of a solve of `cascade` over probes [probeOffset,
 * probeOffset + updatedCount) (mod the probe count) with the current
 * sb_params, exactly as the trace forms them (gi_probes.js:1977-1987): host
 * arrays of updatedCount * raysPerProbe * 3 floats, ray slot * rays + k. A
 * read-back seam for checks (the reference's _debugRead, 4830-4841).
 * Synchronizes. */
sb_status sb_probe_rays(sb_ctx* ctx, uint32_t cascade, uint32_t probeOffset, uint32_t updatedCount, float* roOut,
                        float* rdOut);

/* ---------------------------------------------------- BLAS build (GPU) */

/* BLAS build on the GPU, replacing the CPU MeshBVH build + flattenBVHRoot of
 * each mesh (spectral_scene.js:898-966, 658-721): a linear BVH over the
 * triangles' bounds centres (30-bit Morton codes, stable radix sort, binary
 * radix tree), collapsed to leaves of at most `leafSize` (1..255) triangles,
 * emitted in the reference's threaded layout: 8 x u32 per node, pre-order
 * with the left child at i+1, miss = first node after the subtree, payload
 * (count << 24 | first position) or 0xFFFFFFFF; node bounds are the exact
 * min/max of their triangles' vertices (what a refit gives). triOrderOut[i] =
 * the source triangle at BVH position i; miss links and leaf offsets are
 * relative to this BLAS, as sbh_build_blas's. The tree differs from MeshBVH's
 * (LBVH instead of CENTER splits); closest hits are the same up to exact-t
 * ties, as for any valid BVH.
 * sb_build_blas_device: positions (vertexCount x 3 f32) and indices (triCount x
 * 3 u32) are device arrays; nodesOut (2 * triCount x 8 u32), triOrderOut and
 * nodeCountOut (1 u32) device outputs; enqueued on the context's stream, an
 * out-of-range index is reported by sb_synchronize (SB_ERR_LAYOUT_VIOLATION).
 * sb_build_blas_gpu: the same with host arrays in and out (index range
 * checked first); synchronizes. */
sb_status sb_build_blas_device(sb_ctx* ctx, const float* positions, uint32_t vertexCount, const uint32_t* indices,
                               uint32_t triCount, uint32_t leafSize, uint32_t* nodesOut, uint32_t* triOrderOut,
                               uint32_t* nodeCountOut);
sb_status sb_build_blas_gpu(sb_ctx* ctx, const float* pos3, uint32_t vertexCount, const uint32_t* index3,
                            uint32_t triCount, uint32_t leafSize, uint32_t* nodesOut, uint32_t* triOrderOut,
                            uint32_t* nodeCountOut);

/* Fine-cascade placement (fitFineBox, gi_probes.js:2963-3030): over the coarse
 * box (boxMin, boxSize: the Box3 min and getSize() of C0's grid, doubles), a
 * 16^3 histogram of the pooled triangles' centroids (the pool's vertexData as
 * uploaded, as the reference bins it), the bins of >= 0.4 x the peak united,
 * padded by one bin, each axis clamped to [0.25, 0.60] of the coarse box and
 * moved inside it. *found = 0 when the histogram is empty or the cluster spans
 * the whole box (the reference then places no C1). The histogram runs on the
 * GPU; synchronizes. */
sb_status sb_fit_fine_box(sb_ctx* ctx, const double boxMin[3], const double boxSize[3], double outMin[3],
                          double outSize[3], int32_t* found);

/* ------------------------------------------------------- receiver gather */

/* The receiver's uniforms (GiProbeNode, gi_probes.js:306-358). */
typedef struct sb_gather_params {
    float normalBias[2];       /* sample-point offset along the stable normal; the
                                  point uses normalBias[0] for both cascades, as
                                  GiProbeNode.setup does (0.04)                   */
    float chebyBias[2];        /* Chebyshev depth tolerance per cascade (0)       */
    float chebyStrength;       /* 0 = pure trilinear (default), 1 = full
                                  Chebyshev visibility and wrap weights           */
    float detailStrength;      /* dual-detail blend toward the detail normal (1)  */
    float intensity;           /* output scale (1)                                */
    float enabled;             /* output gate (1)                                 */
    float samplePositionScale; /* debug position scale (1)                        */
    float sampleBiasScale;     /* debug bias scale (1)                            */
    float borderBand;          /* fine-box blend band as a fraction of it (0.15)  */
    uint32_t cascades;         /* 1: cascade 0 alone; 2: cascade 1 of the context
                                  is the fine box blended inside cascade 0        */
    uint32_t dualDetail;       /* 1: fetch at both normals and blend by
                                  detailStrength (one cascade only)               */
    float reflectionIntensity; /* reflection layer scale, 0..1 (1)                */
    float roughnessLimit;      /* receivers rougher than this get no reflection (1) */
} sb_gather_params;
void sb_gather_params_defaults(sb_gather_params* p);
/* Receiver gather (GiProbeNode.sampleIrradiance and setup, gi_probes.js:530-657,
 * 816-850, 884-928): per G-buffer sample the irradiance of the context's
 * current atlases, E = max(trilinear 8-tap gather, 0) * intensity * enabled.
 * position, stableNormal (the bias / visibility normal) and detailNormal (the
 * fetch direction) are DEVICE arrays of `count` float4 (xyz used, 16-byte
 * aligned), out a device array of `count` float4 (rgb, 1). Enqueued on the
 * context's stream; reads the atlases of the last enqueued solve. Classification
 * is inert (no state atlas); the two-cascade path picks each cage at the
 * unbiased surface position. Errors: SB_ERR_INVALID_ARG (null, misaligned,
 * cascades not 1 or 2, dualDetail with 2 cascades), SB_ERR_NOT_READY (a
 * cascade not configured). */
sb_status sb_gather_irradiance(sb_ctx* ctx, const sb_gather_params* params, const float* position,
                               const float* stableNormal, const float* detailNormal, uint32_t count, float* out);
/* The combined receiver with the reflection lobes (GiProbeNode.
 * sampleIrradianceAndRough / _sampleCombinedCascadeLooped and the reflection
 * branch of setup, gi_probes.js:658-806, 893-925): per sample the irradiance
 * (as sb_gather_irradiance, except that each cage is chosen at the biased
 * point and the fine-box band at the surface position, as that path does)
 * and the local reflection layer. reflection: DEVICE float4 per sample,
 * xyz = the receiver's reflection direction (not necessarily unit), w = its
 * roughness. Per cage tap with a live lobe the reflection ray is intersected
 * with the sphere of the probe's mean depth toward it (parallax), and the rough
 * atlas (and for tiers high / ultra the glossy atlas, blended by
 * smoothstep(0.22, 0.58, roughness)) is fetched in the corrected direction,
 * weighted by the tap weight squared. outReflection = (rgb * rw, coverage * rw)
 * with rw = clamp(reflectionIntensity * enabled * (roughness <= roughnessLimit),
 * 0, 1): the renderer composites radiance * (1 - w) + rgb. Needs a reflection
 * tier other than off (SB_ERR_NOT_READY otherwise). */
sb_status sb_gather_reflections(sb_ctx* ctx, const sb_gather_params* params, const float* position,
                                const float* stableNormal, const float* detailNormal, const float* reflection,
                                uint32_t count, float* outIrradiance, float* outReflection);

/* ------------------------------------------------- refit / TLAS lanes (GPU) */

/* BLAS refit over node range [root, end) from the current vertexData
 * (refitFlatBlasRange, gi_refit.js:34-165): exact min/max, bit-identical to the
 * reference's CPU walk. Layout violations latch SB_ERR_LAYOUT_VIOLATION. */
sb_status sb_refit_blas(sb_ctx* ctx, uint32_t root, uint32_t end);

/* BLAS refit that allocates nothing. No counterpart in the reference.
 * For callers that cannot call cudaMalloc: hosts whose device memory belongs to
 * another allocator (an engine heap or interop pool that hands out only its own
 * buffers), and per-frame paths where an allocation's implicit device-wide
 * synchronisation would stall the frame. sb_create allocates, so this entry
 * point takes no context: the caller passes device pointers to its own node
 * (8 x u32 per node, updated in place), triangle-index (3 x u32) and vertex
 * (8 x f32) buffers. Node bounds over [root, end) come out bit-identical to
 * sb_refit_blas on the same inputs; the pre-gathered triangles of a context are
 * not touched. The refit's scratch (parent links, arrival counters, the layout
 * gate) is one file-scope device array of 2 * SB_REFIT_STATIC_MAX_NODES + 64
 * u32 (4 MiB), held by every device that loads the library until exit; ranges
 * of more than SB_REFIT_STATIC_MAX_NODES nodes return SB_ERR_INVALID_ARG.
 * Every call looks up the array's device address for the current device
 * (cudaGetSymbolAddress, with that device current; the first call on a device
 * may load the library's device code there, so make it before any stream
 * capture), so a cudaDeviceReset that reloads the array is followed. Every
 * call shares the array and clears the part it uses; calls that overlap on the
 * GPU (other streams or host threads) race on it. The call runs on
 * `cuda_stream` (NULL = legacy default stream) and synchronises it to read the
 * gate. Its layout check is stricter than refitFlatBlasRange's: a range whose
 * nodes do not form one tree (a node no parent reaches, or two roots) is
 * refused, where the reference would refit it; the per-BLAS ranges of a pool
 * always form one tree. Errors: SB_ERR_INVALID_ARG, SB_ERR_LAYOUT_VIOLATION
 * (rebuild), SB_ERR_NO_DEVICE, SB_ERR_CUDA; `msg` (may be NULL) receives the
 * text. */
#define SB_REFIT_STATIC_MAX_NODES 524288u
sb_status sb_refit_blas_static(uint32_t* nodes, uint32_t nodeCount, const uint32_t* triIndex,
                               uint32_t triCount, const float* vertexData, uint32_t vertexCount,
                               uint32_t root, uint32_t end, void* cuda_stream, char* msg,
                               size_t msgLen);

/* Deform lane for one BLAS (updateDeforms, spectral_scene.js:1831-1927): writes
 * vertexCount pooled vertices (8 floats each) from vertexStart, then refits the
 * BLAS [root, end) and re-gathers its triangles. The vertices must be the
 * BLAS's own pooled slice. Follow with sb_update_transforms(ctx, NULL, NULL, 0)
 * to carry the new root bounds into the TLAS, as the reference does. */
sb_status sb_update_deform(sb_ctx* ctx, uint32_t vertexStart, uint32_t vertexCount,
                           const float* vertexData, uint32_t root, uint32_t end);
/* The same lane from the mesh's own attribute arrays, as updateDeforms gathers
 * them: positions (3 floats per vertex) and, when not NULL, normals (3 floats
 * per vertex) replace the first six floats of each pooled vertex; the rest of
 * the record (uv) keeps its build-time value, and so do the normals when NULL
 * (spectral_scene.js:1866-1900). The arrays are copied before the call
 * returns, so the caller may reuse them at once. */
sb_status sb_update_deform_xyz(sb_ctx* ctx, uint32_t vertexStart, uint32_t vertexCount,
                               const float* positions, const float* normals, uint32_t root, uint32_t end);

/* Per-source-instance transform table (computeDynamic inputs,
 * spectral_scene.js:1256-1298): column-major 4x4 world matrices in FP64
 * (three's Matrix4.elements), the active flag and the BLAS node range.
 * A matrix holding a NaN or an infinity returns SB_ERR_INVALID_ARG and a BLAS
 * range outside the pool SB_ERR_LAYOUT_VIOLATION, before anything changes. */
sb_status sb_set_instances(sb_ctx* ctx, uint32_t count, const double* world16,
                           const uint8_t* active, const uint32_t* blasRoot,
                           const uint32_t* blasEnd);
/* TLAS build on device (buildTlasRecords, spectral_scene.js:973-1003, and
 * writeDynamic 1339-1366): FP64 instance AABBs, longest-axis median split with a
 * stable FP64-centroid order; writes instance records in slot order, the TLAS
 * tail and liveInstanceBounds. Order and bounds are bit-exact. */
sb_status sb_build_tlas(sb_ctx* ctx);
/* Transform lane (updateTransforms, spectral_scene.js:1402-1514): new world
 * matrices for `count` source instances; rewrites their instance rows and
 * bounds, then refits the frozen TLAS exactly (refitFlatTlasRange /
 * refitFlatTlasDirty, gi_refit.js:245-430). count == 0 with src == NULL re-derives
 * every slot's bounds from the current BLAS roots (rewriteInstanceRows:false).
 * A non-finite matrix or an instance index out of range returns
 * SB_ERR_INVALID_ARG with nothing enqueued. */
sb_status sb_update_transforms(sb_ctx* ctx, const uint32_t* srcInstances, const double* world16,
                               uint32_t count);

/* ------------------------------------------------------ differentiation */

/* Adjoint of shade+blend+upload with hit records and visibility held fixed.
 * Parameters: per-material albedo RGB (material record floats 0..2) and
 * emissive RGB (floats 7..9), and per light a scale s of its record colour
 * (floats 7..9) at s = 1: dIntensity[l] = dL/ds_l, so a light of intensity I
 * has dL/dI = dIntensity[l] / I. Every branch of the forward (clamps, the
 * temporal mix's selects) is held at its recorded side; the RGBA16F rounding
 * of the atlas a later solve reads is passed straight through. */
typedef struct sb_grads {
    float* dAlbedo;      /* materialCount*3 */
    float* dEmissive;    /* materialCount*3 */
    float* dIntensity;   /* lightCount      */
} sb_grads;

/* Differentiable forward: clears the cascade's histories and atlases, then runs
 * `solves` (1..8) feedback solves over all its probes, each a full sb_solve,
 * and records the tape on device: per solve the 16-byte hit records and
 * visibility masks, the history it starts from and the atlas its bounce reads;
 * after the last, the final history and the FP32 upload output E
 * (SB_BUF_RECORD_E). With target != NULL (f32 RGB per interior texel,
 * probe-major, probeTotal*36*3) it also returns the loss
 * sum over the interior irradiance texels of the last solve of (E - target)^2,
 * accumulated in FP64. Synchronizes when target != NULL. */
sb_status sb_forward_record(sb_ctx* ctx, uint32_t cascade, uint32_t solves,
                            const float* target, double* loss);
/* Reverse pass of the last sb_forward_record (which must have had a target):
 * re-shades each solve from its recorded hits and runs the adjoint kernels from
 * the last solve back to the first. Fills the gradients (host pointers; any may
 * be NULL) and synchronizes. SB_ERR_NOT_READY when no tape is recorded or a
 * scene, light, parameter or cascade change happened since it was. */
sb_status sb_backward(sb_ctx* ctx, sb_grads* grads);

/* -------------------------------------------------- graphs and autotuning */

/* The device-side motion lane of one context in a captured frame: BLAS
 * refits of the given node ranges (the deform lane after its vertices are in
 * place), then, with refitTlas, instance bounds from the BLAS roots and the
 * TLAS refit (sb_update_transforms(ctx, NULL, NULL, 0)). */
typedef struct sb_frame_lane {
    sb_ctx* ctx;
    const uint32_t* refitRoots;
    const uint32_t* refitEnds;
    uint32_t refitCount;
    int32_t refitTlas;
} sb_frame_lane;

/* Capture the per-frame chain refit -> TLAS refit -> trace -> shade -> blend
 * of several contexts as one CUDA graph owned by items[0].ctx: every lane a
 * parallel branch, joined ahead of one batched solve of `items` (the kernels
 * of sb_solve_batch). The call runs the frame once as ordinary launches (that
 * run applies host-side effects such as layout checks and queue growth) and
 * captures it; it does not replay it. Synchronizes. */
sb_status sb_graph_capture_batch(const sb_frame_lane* lanes, uint32_t laneCount,
                                 const sb_solve_item* items, uint32_t itemCount);
/* The single-context form: lane (ctx, refit ranges, refitTlas) and one solve. */
sb_status sb_graph_capture_frame(sb_ctx* ctx, uint32_t cascade, uint32_t probeOffset,
                                 uint32_t updatedCount, const uint32_t* refitRoots,
                                 const uint32_t* refitEnds, uint32_t refitCount,
                                 int32_t refitTlas);
/* Replay the frame captured by this context: one cudaGraphLaunch on its
 * stream, after the other member contexts' pending work. Each replay takes the
 * members' current parameters (sb_set_params: jitter, hysteresis, ...),
 * lights, materials and scene-BVH marks. When a member's buffers or layouts
 * changed since the capture (scene / range uploads that repack, instances,
 * TLAS build, cascade configuration, tuning) the frame runs as ordinary
 * launches and is captured again. Member contexts must outlive the graph.
 * sb_get_stats' lastSolveMs then covers the whole frame. Enqueue only. */
sb_status sb_graph_launch(sb_ctx* ctx);
/* Free the captured frame (also done by sb_destroy of the owner). */
sb_status sb_graph_destroy(sb_ctx* ctx);

typedef struct sb_tuning {
    uint32_t traceBlock;      /* threads per block of the trace kernels            */
    uint32_t sortKey;         /* ray issue order: 0 = direction-major (ray k of
                                 neighbouring probes per warp), 1 = probe-major,
                                 2 = direction-major over 4 x 4 x 2 probe tiles
                                 (full updates from probe 0; else as 0),
                                 3 = as 2, with the closest-hit stage's 32-ray
                                 batches issued costliest first, by the cycles
                                 each took in the previous full sb_solve of the
                                 cascade (sb_solve only; batches run as 2). On
                                 the 8-wide tree (bvhKind 1) the closest-hit
                                 stage refills lanes ray by ray, and 3 acts
                                 as 2                                            */
    uint32_t smemTlasNodes;   /* TLAS nodes staged in shared memory (0 = none)     */
    uint32_t bvhKind;         /* scene BVH over (triangle, instance) items, rebuilt
                                 on structural changes: 1 = 8-wide nodes with 8-bit
                                 boxes for closest hits + binary for any hits
                                 (default); 2 = binary only.
                                 0 = the reference's TLAS + BLASes                */
    uint32_t smemWideNodes;   /* bvhKind 1: the first (top-level) 8-wide nodes staged
                                 in shared memory per CTA of the closest-hit stage,
                                 80 bytes each (0 = none, at most 512)             */
} sb_tuning;
sb_status sb_get_tuning(const sb_ctx* ctx, sb_tuning* out);
/* The ray/triangle test this library was built with: 0 = the reference's
 * Moller-Trumbore test (spectral_traverse.js:393-409), the parity default of
 * libspeedball_cuda.so; 1 = the watertight test of Woop, Benthin & Wald 2013
 * (libspeedball_cuda_watertight.so, built with SB_WATERTIGHT=1): no ray passes
 * between two triangles that share an edge or a vertex. Both apply the
 * reference's side and alpha acceptance to the same (u, v, t, det sign). */
uint32_t sb_triangle_test(void);
sb_status sb_set_tuning(sb_ctx* ctx, const sb_tuning* t);
/* Time full solves of `cascade` under candidate tunings (bvhKind 1 / 2 / 0,
 * traceBlock 128 / 192 / 256, sortKey 0-3, for bvhKind 1 smemWideNodes
 * 0 / 73 / 512, and for bvhKind 0 TLAS staging
 * off / 512 nodes), keep the fastest on the context and return it. The
 * cascade's histories and atlases are restored afterwards. Synchronizes. */
sb_status sb_autotune(sb_ctx* ctx, uint32_t cascade, sb_tuning* chosen);
/* The same for a batch: the lead context's traceBlock and sortKey (the batched
 * launches' parameters) timed on sb_solve_batch(items); each context keeps its
 * own bvhKind. Every item's probe state is restored. Synchronizes. */
sb_status sb_autotune_batch(const sb_solve_item* items, uint32_t count, sb_tuning* chosen);

/* Device-side counters of the last solve (rays, shadow rays, node/tri visits). */
typedef struct sb_stats {
    uint64_t primaryRays, shadowRays;
    uint64_t tlasNodeVisits, instanceVisits, blasNodeVisits, triangleTests;
    float lastSolveMs;        /* trace + blend/upload of the last sb_solve (device time) */
    float lastTraceMs;        /* the three trace stages (primary, shadow, shade)          */
    float lastBlendMs;        /* blend + upload kernel alone                              */
    uint64_t kernelLaunches;  /* kernels this library launched, process-wide              */
    float lastPrimaryMs;      /* per stage, for solves that fit one shadow-job chunk: the
                                 closest-hit stage (k_trace_primary)                     */
    float lastShadowMs;
    float lastShadeMs;
    /* the shadow-ray share of the visit counters above */
    uint64_t shadowTlasNodeVisits, shadowInstanceVisits, shadowBlasNodeVisits, shadowTriangleTests;
    float lastForwardRecordMs;  /* device time of the last sb_forward_record (all solves + loss) */
    float lastBackwardMs;       /* device time of the last sb_backward                       */
    uint64_t sceneBvhBuilds;    /* host builds of the scene BVH (bvhKind 1, 2) so far        */
    uint32_t sceneBvhActive;    /* 1 while the scene BVH answers the walks; 0 while the
                                   reference's TLAS + BLAS walk does (bvhKind 0, or more
                                   than 256 instance slots moved since the last build)       */
    float lastSceneBvhBuildMs;  /* host time of the last scene-BVH build                     */
    float lastEmitMs;           /* the emission stage (k_emit: hit frames, light gates, jobs) */
    uint32_t sceneBvhBuilding;  /* 1 while a background scene-BVH build runs                 */
} sb_stats;
sb_status sb_get_stats(sb_ctx* ctx, sb_stats* out);
/* Rebuild the scene BVH over the current instance placements before the next
 * trace (the reference rebuilds its BVHs only in an idle-gated rebuild,
 * gi_probes.js:3269-3455). Moved instances stay correct without it: up to 256
 * moved slots are walked through their own BLAS, beyond that the reference's
 * two-level walk, refit on the GPU every frame, answers until a rebuild. */
sb_status sb_rebuild_scene_bvh(sb_ctx* ctx);
/* How a scene-BVH rebuild runs (a structural change, or sb_rebuild_scene_bvh).
 * BLOCKING (default): the next trace reads the scene back, builds the trees on
 * the host and uploads them before it runs. BACKGROUND: the next trace reads
 * the scene back and starts the build on a host thread; traces meanwhile use
 * the reference's two-level walk (GPU-refit TLAS + BLASes), and the first trace
 * after the build finished installs the tree, marking the slots that moved or
 * were refit since it read the scene. A build overtaken by another structural
 * change is dropped and the next trace starts a new one. Back in BLOCKING mode,
 * the next trace waits for a build still running. The scene-BVH walks
 * and the two-level walk agree on hit IDs up to near-ties (the parity bar), so
 * a solve's results do not depend on which one answered beyond that. */
enum { SB_SCENE_BVH_BLOCKING = 0, SB_SCENE_BVH_BACKGROUND = 1 };
sb_status sb_set_scene_bvh_build_mode(sb_ctx* ctx, uint32_t mode);
/* Waits for a running background build and installs it (drops it when the
 * scene changed structurally since it started). No-op when none runs. */
sb_status sb_finish_scene_bvh(sb_ctx* ctx);
/* Counting costs a few percent; off by default. */
sb_status sb_enable_counters(sb_ctx* ctx, int32_t on);

#ifdef __cplusplus
}
#endif
#endif /* SPEEDBALL_CUDA_H */
