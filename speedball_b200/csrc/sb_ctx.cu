// sb_ctx.cu — the C ABI (include/speedball_cuda.h): context lifetime, scene and
// light uploads in the reference layouts, cascade configuration, solves, the
// refit / TLAS lanes and read-back. Host code; all device work is enqueued on
// the context's stream.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "sb_flat_scene.cuh"
#include "sb_kernels.cuh"

using namespace sb;

namespace sb {
static std::atomic<uint64_t> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace sb

namespace {

struct Cascade {
    sb_grid grid{};
    bool configured = false;
    uint32_t probeTotal = 0, atlasW = 0, atlasH = 0;
    float4* irr = nullptr;
    float2* depth = nullptr;
    uint2* atlas = nullptr;
    uint2* depthAtlas = nullptr;
    float4* rayData = nullptr;
    uint4* hits = nullptr;
    uint4* vis = nullptr;
    size_t rayCap = 0;
    uint32_t* tileOrder = nullptr;  // probe index per issue position in 4 x 4 x 2 tiles (sortKey 2)
    // sortKey 3: cycles per 32-ray closest-hit batch of the last full solve, and the batch
    // order (costliest first) built from them; ready once a full solve has recorded costs
    uint32_t* batchCost = nullptr;
    uint32_t* batchOrder = nullptr;
    size_t batchCap = 0;
    bool batchOrderReady = false;
    float* emitterVis = nullptr;  // probeTotal x 16 emitter visibility history
    // reflection lobes, allocated for reflTier (sb_set_reflection_quality)
    uint32_t reflTier = 0;
    float4* roughSpec = nullptr;
    uint2* roughAtlas = nullptr;
    float4* glossyNum = nullptr;
    float* glossyDen = nullptr;
    uint2* glossyAtlas = nullptr;
    uint32_t glossyOct = 1, glossyTile = 1, glossyInterval = 0, glossyPhase = 0;
    uint32_t glossyTilesX = 1, glossyTilesY = 1;
};

}  // namespace

struct sb_ctx {
    int device = 0;
    uint32_t flags = 0;
    uint32_t walkStepLimit = 0;  // sb_set_walk_step_limit (0 = the defaults)
    BlasBuilder* builder = nullptr;  // GPU BLAS build scratch (sb_build_blas_*)
    uint32_t* dHist = nullptr;       // sb_fit_fine_box's 16^3 histogram
    cudaStream_t stream = nullptr;
    cudaStream_t ownStream = nullptr;
    std::string err;
    int numSms = 148;

    SceneBuffers B;
    bool sceneLoaded = false;
    bool needPack = false;     // full validation + derived re-pack before the next solve
    bool tlasPending = false;  // TLAS tail must be built on device (sb_build_tlas)
    bool tlasOnDevice = false; // the TLAS (and its slot maps) came from sb_build_tlas
    size_t cap[6] = {0, 0, 0, 0, 0, 0};  // element capacities of the six scene buffers

    InstanceTable I;
    bool instancesSet = false;
    uint32_t* instOwner = nullptr;
    uint32_t* dStage = nullptr;   // staging for src lists
    // sb_update_deform_xyz: page-locked and device staging of positions + normals,
    // and the event after the copy that last read the page-locked buffer
    float* hDeform = nullptr;
    float* dDeform = nullptr;
    size_t deformCap = 0;  // floats
    cudaEvent_t evDeform = nullptr;
    bool deformPending = false;
    double* dStageM = nullptr;    // staging for matrices
    size_t stageCap = 0;

    uint32_t* dErr = nullptr;
    uint32_t* dGate = nullptr;     // 16 layout verdicts, one per cached refit range, then their 16 subtree counts
    // Refit ranges whose parent links and layout checks are current: valid while
    // packEpoch is unchanged (no upload touched nodes, indices or materials since).
    struct RefitRange { uint32_t root = 0, end = 0, epoch = 0; bool used = false; };
    RefitRange refitRanges[16];
    uint32_t packEpoch = 1, refitNext = 0;
    uint32_t* dWork = nullptr;
    unsigned long long* dCounters = nullptr;
    bool countersOn = false;

    Cascade casc[SB_MAX_CASCADES];
    sb_params params{};
    uint32_t lightCount = 0, emitterBase = 0, emitterCount = 0;
    uint32_t reflectTier = 0;  // sb_set_reflection_quality
    int32_t clustered = 0;
    bool lightGridDirty = false;
    bool lightGatesDirty = false;  // the gate table lags the light records
    std::vector<float> hostLights;

    // 512 TLAS nodes = 32 KB of child pairs per CTA; probe-tile issue order with the closest-hit
    // batches costliest first (atrium solve 0.400 -> 0.387 ms against tile order alone)
    TraceTuning tune{256u, 512u, 3u, 148};
    uint32_t bvhKind = 1;          // 1 = scene BVH, 8-wide for closest hits (default); 2 = binary scene
                                   // BVH only; 0 = the reference's TLAS + BLASes (sb_flat.h)
    FlatScene flat;
    float4* jobs = nullptr;        // shadow-ray job queue (2 float4 per job)
    uint32_t jobCap = 0;
    cudaEvent_t ev0 = nullptr, evMid = nullptr, ev1 = nullptr, evA = nullptr, evB = nullptr, evC = nullptr;
    cudaEvent_t syncEv = nullptr;  // cross-context ordering of batched solves
    bool timed = false;
    bool lastWasGraph = false;     // ev0..ev1 bracket a graph launch (whole frame, no stage events)
    bool singleChunk = true;
    bool capturing = false;        // enqueueing into a CUDA graph capture: no timing events

    // Buffers, layouts and configuration a captured graph refers to: bumped by
    // every call that may reallocate or re-lay them out.
    uint64_t structGen = 1;
    // The per-frame CUDA graph this context owns (sb_graph_capture_*).
    struct Graph {
        struct Lane {
            sb_ctx* ctx;
            std::vector<uint32_t> roots, ends;
            int32_t refitTlas;
        };
        std::vector<Lane> lanes;
        std::vector<sb_solve_item> items;
        std::vector<std::pair<sb_ctx*, std::pair<uint64_t, uint32_t>>> keys;  // (structGen, packEpoch) per context
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t nodes[5] = {};        // the batched kernels, in stage order
        cudaKernelNodeParams params[5] = {};
        std::vector<cudaStream_t> branches;   // one per lane while capturing
        std::vector<cudaEvent_t> joins;
        cudaEvent_t fork = nullptr;
        uint32_t kernelNodes = 0;             // kernels one replay launches
        bool timed = false;
    } graph;

    // Differentiable solves (sb_forward_record / sb_backward). `epoch` counts
    // changes to anything the shading reads; a tape is only replayed under the
    // epoch it was recorded in.
    uint64_t epoch = 1;
    float4* recordE = nullptr;     // set while a recorded solve runs: FP32 upload output
    struct Tape {
        uint32_t cascade = 0, solves = 0, probes = 0, rays = 0, texels = 0;
        uint64_t epoch = 0;
        bool ready = false, hasTarget = false, timedF = false, timedB = false;
        uint4* hits = nullptr; size_t hitsCap = 0;       // solves x probes x rays
        uint4* vis = nullptr; size_t visCap = 0;
        float4* hist = nullptr; size_t histCap = 0;      // (solves + 1) x probes x 64: history before each solve
        uint2* atlas = nullptr; size_t atlasCap = 0;     // solves x texels: the atlas each solve's bounce reads
        float4* E = nullptr; size_t ECap = 0;            // probes x 36: last solve's upload output
        float4* gE = nullptr; size_t gECap = 0;
        float* target = nullptr; size_t targetCap = 0;   // probes x 36 x 3
        float4* shaded = nullptr; size_t shadedCap = 0;  // probes x rays: re-shaded radiance
        float4* gR = nullptr; size_t gRCap = 0;
        float4* gH = nullptr; size_t gHCap = 0;          // 2 x probes x 64 (ping-pong)
        float4* gA = nullptr; size_t gACap = 0;          // 2 x texels (ping-pong)
        double* gParam = nullptr; size_t gParamCap = 0;  // materials x 6 + lights
        double* loss = nullptr; size_t lossCap = 0;
        cudaEvent_t evF0 = nullptr, evF1 = nullptr, evB0 = nullptr, evB1 = nullptr;
    } tape;
};

namespace {

sb_status fail(sb_ctx* c, sb_status s, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
sb_status fail(sb_ctx* c, sb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return s;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? SB_ERR_OOM : SB_ERR_CUDA, "%s: %s", \
                        #call, cudaGetErrorString(e_));                                          \
    } while (0)

template <class T> cudaError_t grow(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}
template <class T> void release(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

constexpr uint64_t kJobCapMax = 64ull << 20;  // 64 Mi shadow jobs (2 GiB) per trace chunk

uint32_t tlas_nodes_for(uint32_t n) {
    // node count of the median split with leaf size 2 (buildTlasRecords)
    if (n == 0) return 0;
    std::vector<uint32_t> t(n + 1);
    t[0] = 1;
    for (uint32_t m = 1; m <= n; ++m) t[m] = m <= 2 ? 1u : 1u + t[m >> 1] + t[m - (m >> 1)];
    return t[n];
}

DevScene dev_scene(const sb_ctx* c) {
    DevScene S;
    S.nodes = reinterpret_cast<const uint4*>(c->B.nodes);
    S.tris = c->B.tris;
    S.triMaterial = c->B.triMaterial;
    S.materials = c->B.materials;
    S.inst = c->B.inst;
    S.tlas = c->B.tlas;
    S.lights = c->B.lights;
    S.lightGates = c->B.lightGates;
    S.triIndex = c->B.triIndex;
    S.vertexData = c->B.vertexData;
    S.pairs = c->B.pairs;
    S.tlasPairs = c->B.tlasPairs;
    S.depth = c->B.depth;
    c->flat.fill(S);
    S.slotBounds = c->instancesSet && c->tlasOnDevice ? c->I.liveBounds : nullptr;
    S.nodeCount = c->B.nodeCount;
    S.triCount = c->B.triCount;
    S.instCount = c->B.instCount;
    S.tlasNodeCount = c->B.tlasNodeCount;
    S.materialCount = c->B.materialCount;
    S.lightCount = c->lightCount;
    S.clustered = c->clustered;
    S.valid = c->B.valid;
    S.iterCap = c->walkStepLimit ? c->walkStepLimit : SB_WALK_STEPS_DEFAULT;
    S.iterCapRef = c->walkStepLimit ? c->walkStepLimit : SB_WALK_STEPS_REF_DEFAULT;
    return S;
}

void fill_grid(DevCascade& D, const sb_grid& g) {
    for (int a = 0; a < 3; ++a) {
        D.gridMin[a] = g.gridMin[a];
        D.gridSize[a] = g.gridSize[a];
        D.res[a] = g.res[a];
    }
    D.rays = g.raysPerProbe;
    D.maxDist = g.maxDist;
    D.cellMin = g.cellMin;
    D.probeTotal = g.res[0] * g.res[1] * g.res[2];
    D.atlasW = g.res[0] * 8u;
    D.atlasH = g.res[1] * g.res[2] * 8u;
}

DevCascade dev_cascade(const sb_ctx* c, uint32_t ci, uint32_t probeOffset, uint32_t updated) {
    const Cascade& K = c->casc[ci];
    DevCascade D{};
    fill_grid(D, K.grid);
    const sb_grid& g0 = c->casc[0].configured ? c->casc[0].grid : K.grid;
    for (int a = 0; a < 3; ++a) {
        D.g0Min[a] = g0.gridMin[a];
        D.g0Size[a] = g0.gridSize[a];
        D.g0Res[a] = g0.res[a];
    }
    D.probeOffset = probeOffset;
    D.updatedCount = updated;
    D.rayData = K.rayData;
    D.hits = K.hits;
    D.vis = K.vis;
    D.irr = K.irr;
    D.depth = K.depth;
    D.atlasPrev = K.atlas;
    D.atlas = K.atlas;
    D.depthAtlas = K.depthAtlas;
    D.eOut = c->recordE;
    D.lights = c->B.lights;
    D.emitterBase = c->emitterBase;
    D.emitterCount = c->emitterCount;
    D.emitterVis = K.emitterVis;
    D.reflect = K.reflTier;
    D.roughSpec = K.roughSpec;
    D.roughAtlas = K.roughAtlas;
    D.glossyNum = K.glossyNum;
    D.glossyDen = K.glossyDen;
    D.glossyAtlas = K.glossyAtlas;
    D.glossyOct = K.glossyOct;
    D.glossyTile = K.glossyTile;
    D.glossyInterval = K.glossyInterval;
    D.glossyPhase = K.glossyPhase;
    D.glossyTilesX = K.glossyTilesX;
    D.glossyAtlasW = K.glossyTilesX * K.glossyTile;
    return D;
}

// The reflection buffers of one cascade for ctx->reflectTier
// (REFLECTION_QUALITY_TIERS, gi_probes.js:60-65; glossy tiles and their packing
// 970-975, 3103-3110), all cleared: histories and supports to 0, the rough
// and glossy atlases to vec4(0) (clearAtlasKernel / clearGlossyAtlasKernel,
// 2703-2724). The glossy phase restarts at 0.
sb_status alloc_reflection(sb_ctx* ctx, Cascade& K) {
    release(K.roughSpec); release(K.roughAtlas); release(K.glossyNum); release(K.glossyDen);
    release(K.glossyAtlas);
    const uint32_t tier = ctx->reflectTier, P = K.probeTotal;
    K.reflTier = tier;
    K.glossyPhase = 0;
    K.glossyOct = tier == SB_REFLECT_HIGH ? 8u : tier == SB_REFLECT_ULTRA ? 16u : 1u;
    K.glossyTile = tier >= SB_REFLECT_HIGH ? K.glossyOct + 2u : 1u;
    K.glossyInterval = tier == SB_REFLECT_HIGH ? 2u : tier == SB_REFLECT_ULTRA ? 1u : 0u;
    K.glossyTilesX = tier >= SB_REFLECT_HIGH ? std::max(1u, (uint32_t)std::ceil(std::sqrt((double)P))) : 1u;
    K.glossyTilesY = tier >= SB_REFLECT_HIGH ? std::max(1u, (P + K.glossyTilesX - 1) / K.glossyTilesX) : 1u;
    if (tier == SB_REFLECT_OFF || P == 0) return SB_OK;
    size_t c = 0;
    const size_t texels = (size_t)P * 64u;
    CK(grow(K.roughSpec, c, texels)); c = 0;
    CK(grow(K.roughAtlas, c, texels)); c = 0;
    CK(cudaMemsetAsync(K.roughSpec, 0, texels * sizeof(float4), ctx->stream));
    CK(cudaMemsetAsync(K.roughAtlas, 0, texels * sizeof(uint2), ctx->stream));
    if (tier >= SB_REFLECT_HIGH) {
        const size_t gt = (size_t)P * K.glossyTile * K.glossyTile;
        const size_t ga = (size_t)K.glossyTilesX * K.glossyTile * K.glossyTilesY * K.glossyTile;
        CK(grow(K.glossyNum, c, gt)); c = 0;
        CK(grow(K.glossyDen, c, gt)); c = 0;
        CK(grow(K.glossyAtlas, c, ga)); c = 0;
        CK(cudaMemsetAsync(K.glossyNum, 0, gt * sizeof(float4), ctx->stream));
        CK(cudaMemsetAsync(K.glossyDen, 0, gt * sizeof(float), ctx->stream));
        CK(cudaMemsetAsync(K.glossyAtlas, 0, ga * sizeof(uint2), ctx->stream));
    }
    return SB_OK;
}

sb_status pack_if_needed(sb_ctx* ctx) {
    if (!ctx->needPack) return SB_OK;
    if (ctx->capturing) return fail(ctx, SB_ERR_NOT_READY, "a re-pack cannot run inside a graph capture");
    ++ctx->packEpoch;  // cached refit verdicts refer to the old layout
    uint32_t one = 1u;
    CK(cudaMemcpyAsync(ctx->B.valid, &one, 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_pack_scene(ctx->B, ctx->dErr, ctx->stream));
    if (!ctx->tlasPending && ctx->B.tlasNodeCount && ctx->instancesSet)
        CK(launch_tlas_index(ctx->B, ctx->I, ctx->instOwner, ctx->dErr, ctx->stream));
    ctx->needPack = false;
    return SB_OK;
}

// The scene BVH of bvhKind 1 and 2: rebuilt after structural changes, marks of
// moved slots uploaded. A build that cannot serve (too deep, too large) leaves
// the reference two-level walk in use.
sb_status flat_if_needed(sb_ctx* ctx) {
    ctx->flat.enabled = ctx->bvhKind == 1 || ctx->bvhKind == 2;
    ctx->flat.wide = ctx->bvhKind == 1;
    std::string why;
    const bool order = ctx->tlasOnDevice && ctx->instancesSet;
    CK(ctx->flat.prepare(ctx->B, order ? ctx->I.order : nullptr, order ? ctx->I.count : 0u, ctx->stream, why));
    return SB_OK;
}

sb_status light_grid_if_needed(sb_ctx* ctx) {
    if (ctx->lightGatesDirty) {  // the emission stage's gate table, from the current records
        size_t cap = ctx->B.lightGates ? 64u * 3u : 0u;
        CK(grow(ctx->B.lightGates, cap, (size_t)64 * 3));
        CK(launch_light_gates(ctx->B.lights, ctx->B.lightGates, ctx->stream));
        ctx->lightGatesDirty = false;
    }
    if (!ctx->lightGridDirty || !ctx->clustered || !ctx->casc[0].configured) return SB_OK;
    DevCascade g0{};
    fill_grid(g0, ctx->casc[0].grid);
    CK(launch_light_grid(ctx->B.lights, ctx->lightCount, g0, ctx->stream));
    ctx->lightGridDirty = false;
    return SB_OK;
}

// A material-buffer range that lies inside the material records and writes
// none of the fields the packer reads (opacity 10, side 22, alpha test 23,
// flags 26): the derived layouts and the scene BVH stay valid.
bool shading_only(const SceneBuffers& B, uint32_t start, uint32_t count) {
    const uint64_t end = (uint64_t)start + count;
    if (end > (uint64_t)B.materialCount * SB_MAT_STRIDE) return false;
    for (uint64_t i = start; i < end; ++i) {
        const uint32_t f = (uint32_t)(i % SB_MAT_STRIDE);
        if (f == 10 || f == 22 || f == 23 || f == 26) return false;
    }
    return true;
}

sb_status check_grid(sb_ctx* ctx, const sb_grid* g) {
    if (!g) return fail(ctx, SB_ERR_INVALID_ARG, "grid is null");
    for (int a = 0; a < 3; ++a)
        if (g->res[a] < 2 || g->res[a] > 32) return fail(ctx, SB_ERR_INVALID_ARG, "res[%d]=%u outside [2,32]", a, g->res[a]);
    if (g->raysPerProbe < 32 || g->raysPerProbe > 256 || g->raysPerProbe % 16)
        return fail(ctx, SB_ERR_INVALID_ARG, "raysPerProbe=%u: must be 32..256 in steps of 16", g->raysPerProbe);
    return SB_OK;
}

}  // namespace

extern "C" {

uint32_t sb_abi_version(void) { return SB_ABI_VERSION; }

void sb_params_defaults(sb_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->frameJitter = 0.0f;
    p->emitterVisSeed = 0.0f;
    p->hysteresis = 0.60f;              // JITTER_HYSTERESIS_DEFAULTS.gated
    p->hysteresisExponent = 1.0f;
    p->depthSharpness = 7.0f;
    p->radianceClamp = 8.0f;
    p->classifyStrength = 0.0f;
    p->filterStrength = 1.0f;
    p->filterSmooth = 0.5f;
    p->tempChangeSigma1 = 2.5f;
    p->tempChangeHDrop = 0.30f;
    p->tempClampSigma = 6.0f;
    p->nirGate = 0.0f;
    p->nirGain = 1.0f;
    p->skyIntensity = 1.0f;
    p->debugTraceBiasScale = p->debugRayEpsScale = p->debugDirectScale = p->debugEmissiveScale = 1.0f;
    p->debugAlbedoScale = p->debugBounceScale = p->debugCosinePower = 1.0f;
    p->debugTempNoiseHBoost = 0.25f;
    p->debugTempChangeSigma0 = 0.75f;
    p->debugTempMinChangeH = 0.55f;
    p->debugTempVarEps = 0.000025f;
    p->debugTempVarRel = 0.0025f;
    p->debugDepthHistoryScale = 1.0f;
    p->debugFilterKScale = p->debugFilterRelScale = p->debugFilterEpsScale = 1.0f;
}

sb_status sb_create(const sb_device_opts* opts, sb_ctx** out) {
    if (!out) return SB_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return SB_ERR_NO_DEVICE;
    sb_ctx* ctx = new sb_ctx();
    ctx->device = opts ? opts->device : 0;
    ctx->flags = opts ? opts->flags : 0;
    if (ctx->device < 0 || ctx->device >= n) {
        delete ctx;
        return SB_ERR_INVALID_ARG;
    }
    sb_status st = SB_OK;
    do {
        if (cudaSetDevice(ctx->device) != cudaSuccess) { st = SB_ERR_CUDA; break; }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) { st = SB_ERR_CUDA; break; }
        if (prop.major < 10) { st = SB_ERR_UNSUPPORTED; break; }  // sm_100a build
        ctx->numSms = prop.multiProcessorCount;
        ctx->tune.numSms = ctx->numSms;
        if (cudaStreamCreateWithFlags(&ctx->ownStream, cudaStreamNonBlocking) != cudaSuccess) { st = SB_ERR_CUDA; break; }
        ctx->stream = ctx->ownStream;
        if (cudaMalloc(&ctx->dErr, 4) != cudaSuccess || cudaMalloc(&ctx->dGate, 32 * 4) != cudaSuccess ||
            cudaMalloc(&ctx->dWork, 64) != cudaSuccess || cudaMalloc(&ctx->dCounters, 16 * 8) != cudaSuccess ||
            cudaMalloc(&ctx->B.valid, 4) != cudaSuccess || cudaMalloc(&ctx->B.depth, 8) != cudaSuccess) {
            st = SB_ERR_OOM;
            break;
        }
        cudaMemset(ctx->dErr, 0, 4);
        cudaMemset(ctx->B.valid, 0, 4);
        cudaMemset(ctx->B.depth, 0xFF, 8);
        cudaMemset(ctx->dCounters, 0, 128);
        cudaEventCreate(&ctx->ev0);
        cudaEventCreate(&ctx->evMid);
        cudaEventCreate(&ctx->ev1);
        cudaEventCreate(&ctx->evA);
        cudaEventCreate(&ctx->evB);
        cudaEventCreate(&ctx->evC);
        sb_params_defaults(&ctx->params);
        if (cudaDeviceSynchronize() != cudaSuccess) { st = SB_ERR_CUDA; break; }
    } while (0);
    if (st != SB_OK) {
        sb_destroy(ctx);
        return st;
    }
    *out = ctx;
    return SB_OK;
}

void sb_destroy(sb_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    SceneBuffers& B = ctx->B;
    release(B.nodes); release(B.triIndex); release(B.vertexData); release(B.triMaterial); release(B.materials);
    release(B.lights); release(B.lightGates); release(B.tris); release(B.inst); release(B.tlas); release(B.matBits); release(B.parent);
    release(B.arrive); release(B.subRoots); release(B.valid); release(B.pairs); release(B.tlasPairs); release(B.depth);
    ctx->flat.release();
    if (ctx->builder) {
        blas_builder_destroy(ctx->builder);
        ctx->builder = nullptr;
    }
    release(ctx->dHist);
    InstanceTable& I = ctx->I;
    release(I.world); release(I.active); release(I.blasRoot); release(I.blasEnd); release(I.aabb); release(I.invRows);
    release(I.detSign); release(I.order); release(I.slotOf); release(I.liveBounds); release(I.nodeDepth);
    release(I.scratch); release(ctx->instOwner); release(ctx->dStage); release(ctx->dStageM);
    for (auto& K : ctx->casc) {
        release(K.irr); release(K.depth); release(K.atlas); release(K.depthAtlas); release(K.rayData); release(K.hits);
        release(K.emitterVis);
        release(K.tileOrder); release(K.batchCost); release(K.batchOrder);
        release(K.vis);
        release(K.roughSpec); release(K.roughAtlas); release(K.glossyNum); release(K.glossyDen);
        release(K.glossyAtlas);
    }
    release(ctx->jobs);
    auto& G = ctx->graph;
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.graph) cudaGraphDestroy(G.graph);
    for (cudaStream_t s : G.branches) cudaStreamDestroy(s);
    for (cudaEvent_t e : G.joins) cudaEventDestroy(e);
    if (G.fork) cudaEventDestroy(G.fork);
    auto& T = ctx->tape;
    release(T.hits); release(T.vis); release(T.hist); release(T.atlas); release(T.E); release(T.gE);
    release(T.target); release(T.shaded); release(T.gR); release(T.gH); release(T.gA); release(T.gParam);
    release(T.loss);
    for (cudaEvent_t e : {T.evF0, T.evF1, T.evB0, T.evB1})
        if (e) cudaEventDestroy(e);
    release(ctx->dErr); release(ctx->dGate); release(ctx->dWork); release(ctx->dCounters);
    if (ctx->syncEv) cudaEventDestroy(ctx->syncEv);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->evMid) cudaEventDestroy(ctx->evMid);
    if (ctx->evA) cudaEventDestroy(ctx->evA);
    if (ctx->evB) cudaEventDestroy(ctx->evB);
    if (ctx->evC) cudaEventDestroy(ctx->evC);
    if (ctx->evDeform) cudaEventDestroy(ctx->evDeform);
    if (ctx->hDeform) cudaFreeHost(ctx->hDeform);
    if (ctx->dDeform) cudaFree(ctx->dDeform);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->ownStream) cudaStreamDestroy(ctx->ownStream);
    delete ctx;
}

const char* sb_last_error(const sb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

sb_status sb_host_alloc(size_t bytes, void** out) {
    if (!out || bytes == 0) return SB_ERR_INVALID_ARG;
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        *out = nullptr;
        return e == cudaErrorMemoryAllocation ? SB_ERR_OOM : SB_ERR_CUDA;
    }
    return SB_OK;
}

void sb_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

sb_status sb_set_stream(sb_ctx* ctx, void* s) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ctx->stream = s ? (cudaStream_t)s : ctx->ownStream;
    return SB_OK;
}

sb_status sb_set_walk_step_limit(sb_ctx* ctx, uint32_t steps) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ctx->walkStepLimit = steps;
    return SB_OK;
}

sb_status sb_synchronize(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    CK(cudaStreamSynchronize(ctx->stream));
    uint32_t e = 0;
    CK(cudaMemcpy(&e, ctx->dErr, 4, cudaMemcpyDeviceToHost));
    if (e) {
        CK(cudaMemset(ctx->dErr, 0, 4));
        if (e & ERR_LAYOUT) return fail(ctx, SB_ERR_LAYOUT_VIOLATION, "device check: threaded-layout or index violation");
        if (e & ERR_WATCHDOG) return fail(ctx, SB_ERR_DEVICE_WATCHDOG, "device check: traversal iteration cap reached");
        if (e & ERR_NAN_KEY) return fail(ctx, SB_ERR_INVALID_ARG, "device check: NaN instance bounds");
        return fail(ctx, SB_ERR_CUDA, "device error word 0x%x", e);
    }
    return SB_OK;
}

sb_status sb_upload_scene(sb_ctx* ctx, const sb_scene_view* v) {
    if (!ctx || !v) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!v->bvhNodes || !v->triIndex || !v->vertexData || !v->triMaterial || !v->materials)
        return fail(ctx, SB_ERR_INVALID_ARG, "null scene array");
    if (v->nodeCount == 0 || v->triCount == 0 || v->vertexCount == 0 || v->materialCount == 0 || v->instCount == 0)
        return fail(ctx, SB_ERR_INVALID_ARG, "empty scene");
    if (v->triCount >= (1u << 24) || v->nodeCount >= (1u << 24))
        return fail(ctx, SB_ERR_INVALID_ARG, "BVH pool exceeds the 24-bit index ceiling");
    if (v->instBase != v->materialCount * SB_MAT_STRIDE)
        return fail(ctx, SB_ERR_INVALID_ARG, "instBase %u != materialCount*28", v->instBase);
    uint32_t tlasBase = v->instBase + v->instCount * SB_MAT_STRIDE;
    if (v->tlasNodeCount && v->tlasBase != tlasBase)
        return fail(ctx, SB_ERR_INVALID_ARG, "tlasBase %u != instBase + instCount*28", v->tlasBase);
    uint32_t tlasNodes = v->tlasNodeCount ? v->tlasNodeCount : tlas_nodes_for(v->instCount);
    size_t matLen = (size_t)tlasBase + (size_t)tlasNodes * SB_TLAS_STRIDE_F32;
    if (v->tlasNodeCount && v->materialsLen < matLen)
        return fail(ctx, SB_ERR_INVALID_ARG, "materialsLen %u < %zu", v->materialsLen, matLen);
    if (!v->tlasNodeCount && v->materialsLen < tlasBase)
        return fail(ctx, SB_ERR_INVALID_ARG, "materialsLen %u < %u", v->materialsLen, tlasBase);
    cudaSetDevice(ctx->device);
    SceneBuffers& B = ctx->B;
    size_t nN = (size_t)v->nodeCount * 8, nT = (size_t)v->triCount * 3, nV = (size_t)v->vertexCount * 8;
    CK(grow(B.nodes, ctx->cap[0], nN));
    CK(grow(B.triIndex, ctx->cap[1], nT));
    CK(grow(B.vertexData, ctx->cap[2], nV));
    CK(grow(B.triMaterial, ctx->cap[3], (size_t)v->triCount));
    CK(grow(B.materials, ctx->cap[4], matLen));
    size_t cTris = 0, cInst = 0, cTlas = 0, cBits = 0, cPar = 0, cArr = 0, cSub = 0, cPairs = 0, cTlasPairs = 0;
    release(B.tris); release(B.inst); release(B.tlas); release(B.matBits); release(B.parent); release(B.arrive);
    release(B.subRoots);
    release(B.pairs); release(B.tlasPairs);
    CK(grow(B.tris, cTris, (size_t)v->triCount * 3));
    CK(grow(B.inst, cInst, (size_t)v->instCount * 4));
    CK(grow(B.tlas, cTlas, (size_t)tlasNodes * 2));
    CK(grow(B.matBits, cBits, (size_t)v->materialCount));
    CK(grow(B.parent, cPar, (size_t)v->nodeCount));
    CK(grow(B.arrive, cArr, (size_t)v->nodeCount));
    CK(grow(B.subRoots, cSub, (size_t)v->nodeCount));
    if (v->nodeCount < PE_BLAS_MAX_NODES) CK(grow(B.pairs, cPairs, (size_t)v->nodeCount * 4));
    CK(grow(B.tlasPairs, cTlasPairs, (size_t)tlasNodes * 4));
    CK(cudaMemsetAsync(B.depth, 0xFF, 8, ctx->stream));  // no pair layout until the pack derives it
    CK(cudaMemcpyAsync(B.nodes, v->bvhNodes, nN * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(B.triIndex, v->triIndex, nT * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(B.vertexData, v->vertexData, nV * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(B.triMaterial, v->triMaterial, (size_t)v->triCount * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(B.materials, 0, matLen * 4, ctx->stream));
    CK(cudaMemcpyAsync(B.materials, v->materials, (v->tlasNodeCount ? matLen : tlasBase) * 4, cudaMemcpyHostToDevice,
                       ctx->stream));
    B.nodeCount = v->nodeCount;
    B.triCount = v->triCount;
    B.vertexCount = v->vertexCount;
    B.materialsLen = (uint32_t)matLen;
    B.materialCount = v->materialCount;
    B.instBase = v->instBase;
    B.instCount = v->instCount;
    B.tlasBase = tlasBase;
    B.tlasNodeCount = tlasNodes;
    ctx->tlasPending = v->tlasNodeCount == 0;
    ctx->tlasOnDevice = false;
    ctx->sceneLoaded = true;
    ctx->flat.invalidate();
    ++ctx->epoch;
    ++ctx->structGen;
    if (ctx->instancesSet && ctx->I.count != v->instCount) ctx->instancesSet = false;
    // validation + derived layouts; a pending TLAS is packed by sb_build_tlas
    uint32_t one = 1u;
    ++ctx->packEpoch;
    CK(cudaMemcpyAsync(B.valid, &one, 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_pack_scene(ctx->tlasPending ? [&] { SceneBuffers t = B; t.instCount = 0; t.tlasNodeCount = 0; return t; }() : B,
                         ctx->dErr, ctx->stream));
    ctx->needPack = false;
    return SB_OK;
}

sb_status sb_upload_range(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count, const void* src) {
    if (!ctx || (!src && count)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    uint32_t buf = which & 0xFFu, ci = which >> 8;
    cudaSetDevice(ctx->device);
    void* dst = nullptr;
    size_t len = 0, esz = 4;
    SceneBuffers& B = ctx->B;
    switch (buf) {
        case SB_BUF_BVH_NODES: dst = B.nodes; len = (size_t)B.nodeCount * 8; break;
        case SB_BUF_TRI_INDEX: dst = B.triIndex; len = (size_t)B.triCount * 3; break;
        case SB_BUF_VERTEX_DATA: dst = B.vertexData; len = (size_t)B.vertexCount * 8; break;
        case SB_BUF_TRI_MATERIAL: dst = B.triMaterial; len = B.triCount; break;
        case SB_BUF_MATERIALS: dst = B.materials; len = B.materialsLen; break;
        case SB_BUF_LIGHTS: dst = B.lights; len = ctx->B.lightsLen; break;
        case SB_BUF_IRRADIANCE_HISTORY:
        case SB_BUF_DEPTH_HISTORY: {
            if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
                return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", ci);
            Cascade& K = ctx->casc[ci];
            dst = buf == SB_BUF_IRRADIANCE_HISTORY ? (void*)K.irr : (void*)K.depth;
            len = (size_t)K.probeTotal * 64 * (buf == SB_BUF_IRRADIANCE_HISTORY ? 4 : 2);
            break;
        }
        case SB_BUF_IRRADIANCE_ATLAS:
        case SB_BUF_DEPTH_ATLAS: {
            if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
                return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", ci);
            Cascade& K = ctx->casc[ci];
            dst = buf == SB_BUF_IRRADIANCE_ATLAS ? (void*)K.atlas : (void*)K.depthAtlas;
            len = (size_t)K.atlasW * K.atlasH * 4;
            esz = 2;
            break;
        }
        default: return fail(ctx, SB_ERR_INVALID_ARG, "buffer %u is not writable", buf);
    }
    if (!dst) return fail(ctx, SB_ERR_NOT_READY, "buffer %u not allocated", buf);
    if ((size_t)start + count > len) return fail(ctx, SB_ERR_INVALID_ARG, "range [%u,+%u) outside %zu", start, count, len);
    CK(cudaMemcpyAsync((char*)dst + (size_t)start * esz, src, (size_t)count * esz, cudaMemcpyHostToDevice, ctx->stream));
    ++ctx->epoch;
    if (buf <= SB_BUF_MATERIALS && !(buf == SB_BUF_MATERIALS && shading_only(B, start, count))) {
        ++ctx->structGen;
        ctx->needPack = true;
        ctx->flat.invalidate();
    }
    if (buf == SB_BUF_LIGHTS && ctx->clustered) ctx->lightGridDirty = true;
    if (buf == SB_BUF_LIGHTS) ctx->lightGatesDirty = true;
    return SB_OK;
}

// Validates a read and enqueues its copy on the context stream.
static sb_status read_enqueue(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count, void* dstHost) {
    if (!ctx || (!dstHost && count)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    uint32_t buf = which & 0xFFu, ci = which >> 8;
    cudaSetDevice(ctx->device);
    const void* srcp = nullptr;
    size_t len = 0, esz = 4;
    SceneBuffers& B = ctx->B;
    Cascade* K = ci < SB_MAX_CASCADES ? &ctx->casc[ci] : nullptr;
    switch (buf) {
        case SB_BUF_BVH_NODES: srcp = B.nodes; len = (size_t)B.nodeCount * 8; break;
        case SB_BUF_TRI_INDEX: srcp = B.triIndex; len = (size_t)B.triCount * 3; break;
        case SB_BUF_VERTEX_DATA: srcp = B.vertexData; len = (size_t)B.vertexCount * 8; break;
        case SB_BUF_TRI_MATERIAL: srcp = B.triMaterial; len = B.triCount; break;
        case SB_BUF_MATERIALS: srcp = B.materials; len = B.materialsLen; break;
        case SB_BUF_LIGHTS: srcp = B.lights; len = B.lightsLen; break;
        case SB_BUF_IRRADIANCE_HISTORY: if (K) { srcp = K->irr; len = (size_t)K->probeTotal * 256; } break;
        case SB_BUF_DEPTH_HISTORY: if (K) { srcp = K->depth; len = (size_t)K->probeTotal * 128; } break;
        case SB_BUF_IRRADIANCE_ATLAS: if (K) { srcp = K->atlas; len = (size_t)K->atlasW * K->atlasH * 4; esz = 2; } break;
        case SB_BUF_DEPTH_ATLAS: if (K) { srcp = K->depthAtlas; len = (size_t)K->atlasW * K->atlasH * 4; esz = 2; } break;
        case SB_BUF_RAY_DATA: if (K) { srcp = K->rayData; len = K->rayCap * 4; } break;
        case SB_BUF_HIT_RECORDS: if (K) { srcp = K->hits; len = K->hits ? K->rayCap * 4 : 0; } break;
        case SB_BUF_VISIBILITY: if (K) { srcp = K->vis; len = K->vis ? K->rayCap * 4 : 0; } break;
        case SB_BUF_TLAS_ORDER: srcp = ctx->I.order; len = ctx->instancesSet ? ctx->I.count : 0; break;
        case SB_BUF_INSTANCE_BOUNDS: srcp = ctx->I.liveBounds; len = ctx->instancesSet ? (size_t)ctx->I.count * 6 : 0; break;
        case SB_BUF_RECORD_E: srcp = ctx->tape.E; len = ctx->tape.ready ? (size_t)ctx->tape.probes * 36 * 4 : 0; break;
        case SB_BUF_EMITTER_VIS: if (K) { srcp = K->emitterVis; len = K->emitterVis ? (size_t)K->probeTotal * EMITTER_CAP : 0; } break;
        case SB_BUF_ROUGH_SPECULAR: if (K) { srcp = K->roughSpec; len = K->roughSpec ? (size_t)K->probeTotal * 256 : 0; } break;
        case SB_BUF_ROUGH_ATLAS: if (K) { srcp = K->roughAtlas; len = K->roughAtlas ? (size_t)K->atlasW * K->atlasH * 4 : 0; esz = 2; } break;
        case SB_BUF_GLOSSY_SPECULAR:
            if (K) { srcp = K->glossyNum; len = K->glossyNum ? (size_t)K->probeTotal * K->glossyTile * K->glossyTile * 4 : 0; }
            break;
        case SB_BUF_GLOSSY_WEIGHT:
            if (K) { srcp = K->glossyDen; len = K->glossyDen ? (size_t)K->probeTotal * K->glossyTile * K->glossyTile : 0; }
            break;
        case SB_BUF_GLOSSY_ATLAS:
            if (K) {
                srcp = K->glossyAtlas;
                len = K->glossyAtlas ? (size_t)K->glossyTilesX * K->glossyTile * K->glossyTilesY * K->glossyTile * 4 : 0;
                esz = 2;
            }
            break;
        default: return fail(ctx, SB_ERR_INVALID_ARG, "unknown buffer %u", buf);
    }
    if (!srcp) return fail(ctx, SB_ERR_NOT_READY, "buffer %u not available", buf);
    if ((size_t)start + count > len) return fail(ctx, SB_ERR_INVALID_ARG, "range [%u,+%u) outside %zu", start, count, len);
    CK(cudaMemcpyAsync(dstHost, (const char*)srcp + (size_t)start * esz, (size_t)count * esz, cudaMemcpyDeviceToHost,
                       ctx->stream));
    return SB_OK;
}

sb_status sb_read_buffer(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count, void* dstHost) {
    sb_status s = read_enqueue(ctx, which, start, count, dstHost);
    if (s != SB_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream));
    return SB_OK;
}

sb_status sb_read_buffer_async(sb_ctx* ctx, uint32_t which, uint32_t start, uint32_t count, void* dstHost) {
    return read_enqueue(ctx, which, start, count, dstHost);
}

sb_status sb_upload_lights(sb_ctx* ctx, const float* records, uint32_t count, uint32_t emitterBase,
                           uint32_t emitterCount, int32_t clustered) {
    if (!ctx || (!records && count)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (count > SB_MAX_LIGHTS) return fail(ctx, SB_ERR_INVALID_ARG, "%u lights > %u", count, SB_MAX_LIGHTS);
    if (emitterCount > EMITTER_CAP) return fail(ctx, SB_ERR_INVALID_ARG, "%u emitters > %u", emitterCount, EMITTER_CAP);
    if (emitterCount && (uint64_t)emitterBase + emitterCount > count)
        return fail(ctx, SB_ERR_INVALID_ARG, "emitter records [%u,+%u) outside the %u records", emitterBase, emitterCount, count);
    for (uint32_t e = 0; e < emitterCount; ++e)
        if (std::fabs(records[(size_t)(emitterBase + e) * SB_LIGHT_STRIDE] - 3.0f) >= 0.5f)
            return fail(ctx, SB_ERR_INVALID_ARG, "record %u in the emitter range is not a giEmitter (type 3)", emitterBase + e);
    cudaSetDevice(ctx->device);
    uint32_t cells = 0;
    if (clustered) {
        if (!ctx->casc[0].configured) return fail(ctx, SB_ERR_NOT_READY, "clustered lights need cascade 0 configured");
        const sb_grid& g = ctx->casc[0].grid;
        cells = (g.res[0] - 1) * (g.res[1] - 1) * (g.res[2] - 1);
    }
    uint32_t len = SB_MAX_LIGHTS * SB_LIGHT_STRIDE + cells * (SB_LIGHTS_PER_CELL + 1);
    ctx->hostLights.assign(len, 0.0f);
    if (count) std::memcpy(ctx->hostLights.data(), records, (size_t)count * SB_LIGHT_STRIDE * 4);
    size_t cap = ctx->cap[5];
    CK(grow(ctx->B.lights, cap, len));
    ctx->cap[5] = cap;
    ctx->B.lightsLen = len;
    CK(cudaMemcpyAsync(ctx->B.lights, ctx->hostLights.data(), (size_t)len * 4, cudaMemcpyHostToDevice, ctx->stream));
    ctx->lightCount = count;
    ctx->emitterBase = emitterBase;
    ctx->emitterCount = emitterCount;
    ctx->clustered = clustered ? 1 : 0;
    ctx->lightGridDirty = ctx->clustered != 0;
    ctx->lightGatesDirty = true;
    ++ctx->epoch;
    return SB_OK;
}

sb_status sb_set_params(sb_ctx* ctx, const sb_params* p) {
    if (!ctx || !p) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (p->classifyStrength != 0.0f)
        return fail(ctx, SB_ERR_UNSUPPORTED, "probe classification / relocation (classifyStrength > 0) is not built");
    ctx->params = *p;
    ++ctx->epoch;
    return SB_OK;
}

sb_status sb_set_reflection_quality(sb_ctx* ctx, uint32_t tier) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    if (tier > SB_REFLECT_ULTRA) return fail(ctx, SB_ERR_INVALID_ARG, "reflection tier %u (off, rough, high, ultra)", tier);
    if (ctx->capturing) return fail(ctx, SB_ERR_NOT_READY, "reflection buffers cannot be reallocated inside a graph capture");
    cudaSetDevice(ctx->device);
    ctx->reflectTier = tier;
    for (auto& K : ctx->casc) {
        if (!K.configured) continue;
        sb_status s = alloc_reflection(ctx, K);
        if (s != SB_OK) return s;
    }
    ++ctx->epoch;
    ++ctx->structGen;
    return SB_OK;
}

sb_status sb_get_reflection_layout(sb_ctx* ctx, uint32_t ci, sb_reflection_layout* out) {
    if (!ctx || !out) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
        return fail(ctx, SB_ERR_INVALID_ARG, "cascade %u is not configured", ci);
    const Cascade& K = ctx->casc[ci];
    out->tier = K.reflTier;
    out->glossyOct = K.reflTier >= SB_REFLECT_HIGH ? K.glossyOct : 0u;
    out->glossyTile = K.reflTier >= SB_REFLECT_HIGH ? K.glossyTile : 0u;
    out->glossyInterval = K.glossyInterval;
    out->glossyTilesX = K.glossyTilesX;
    out->glossyTilesY = K.glossyTilesY;
    out->glossyAtlasW = K.reflTier >= SB_REFLECT_HIGH ? K.glossyTilesX * K.glossyTile : 0u;
    out->glossyAtlasH = K.reflTier >= SB_REFLECT_HIGH ? K.glossyTilesY * K.glossyTile : 0u;
    out->glossyPhase = K.glossyPhase;
    return SB_OK;
}

sb_status sb_configure_cascade(sb_ctx* ctx, uint32_t ci, const sb_grid* g) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    if (ci >= SB_MAX_CASCADES) return fail(ctx, SB_ERR_INVALID_ARG, "cascade %u >= %u", ci, SB_MAX_CASCADES);
    sb_status s = check_grid(ctx, g);
    if (s != SB_OK) return s;
    cudaSetDevice(ctx->device);
    Cascade& K = ctx->casc[ci];
    uint32_t probeTotal = g->res[0] * g->res[1] * g->res[2];
    bool sameDims = K.configured && K.grid.res[0] == g->res[0] && K.grid.res[1] == g->res[1] &&
                    K.grid.res[2] == g->res[2];
    size_t rays = (size_t)probeTotal * g->raysPerProbe;
    if (!sameDims) {
        release(K.irr); release(K.depth); release(K.atlas); release(K.depthAtlas); release(K.tileOrder);
        release(K.emitterVis);
        size_t c = 0;
        CK(grow(K.emitterVis, c, (size_t)probeTotal * EMITTER_CAP)); c = 0;
        CK(cudaMemsetAsync(K.emitterVis, 0, (size_t)probeTotal * EMITTER_CAP * sizeof(float), ctx->stream));
        CK(grow(K.irr, c, (size_t)probeTotal * 64)); c = 0;
        CK(grow(K.depth, c, (size_t)probeTotal * 64)); c = 0;
        CK(grow(K.atlas, c, (size_t)probeTotal * 64)); c = 0;
        CK(grow(K.depthAtlas, c, (size_t)probeTotal * 64)); c = 0;
        // the probes in 4 x 4 x 2 tiles (row-major over tiles, x fastest inside;
        // edge tiles clipped): 32 consecutive entries form one compact block
        std::vector<uint32_t> order;
        order.reserve(probeTotal);
        const uint32_t rx = g->res[0], ry = g->res[1], rz = g->res[2];
        for (uint32_t tz = 0; tz < rz; tz += 2)
            for (uint32_t ty = 0; ty < ry; ty += 4)
                for (uint32_t tx = 0; tx < rx; tx += 4)
                    for (uint32_t z = tz; z < tz + 2 && z < rz; ++z)
                        for (uint32_t y = ty; y < ty + 4 && y < ry; ++y)
                            for (uint32_t x = tx; x < tx + 4 && x < rx; ++x) order.push_back((z * ry + y) * rx + x);
        CK(grow(K.tileOrder, c, (size_t)probeTotal));
        CK(cudaMemcpy(K.tileOrder, order.data(), (size_t)probeTotal * 4, cudaMemcpyHostToDevice));
    }
    if (rays > K.rayCap || !K.rayData) {
        release(K.rayData); release(K.hits); release(K.vis);
        size_t c = 0;
        CK(grow(K.rayData, c, rays));
        c = 0; CK(grow(K.hits, c, rays));
        c = 0; CK(grow(K.vis, c, rays));
        K.rayCap = rays;
    }
    {
        const size_t batches = (rays + 31) / 32;
        size_t c = K.batchCap;
        CK(grow(K.batchCost, c, batches));
        c = K.batchCap;
        CK(grow(K.batchOrder, c, batches));
        K.batchCap = c;
        K.batchOrderReady = false;  // the batches are those of the new grid
        // identity until a solve has ordered them: always a permutation of the batches
        std::vector<uint32_t> iota(batches);
        for (size_t i = 0; i < batches; ++i) iota[i] = (uint32_t)i;
        CK(cudaMemcpy(K.batchOrder, iota.data(), batches * 4, cudaMemcpyHostToDevice));
    }
    K.grid = *g;
    K.probeTotal = probeTotal;
    K.atlasW = g->res[0] * 8;
    K.atlasH = g->res[1] * g->res[2] * 8;
    K.configured = true;
    if (!sameDims || K.reflTier != ctx->reflectTier) {
        s = alloc_reflection(ctx, K);
        if (s != SB_OK) return s;
    }
    K.glossyPhase = 0;  // every rebuild restarts the glossy interleave (gi_probes.js:3162, 3193, 3224)
    ++ctx->epoch;
    ++ctx->structGen;
    if (!sameDims) {
        DevCascade D = dev_cascade(ctx, ci, 0, 0);
        CK(launch_clear_cascade(D, ctx->stream));
    }
    if (ci == 0 && ctx->clustered) {
        // the cell lists follow C0's grid: re-size the light arena
        const sb_grid& gg = ctx->casc[0].grid;
        uint32_t cells = (gg.res[0] - 1) * (gg.res[1] - 1) * (gg.res[2] - 1);
        uint32_t len = SB_MAX_LIGHTS * SB_LIGHT_STRIDE + cells * (SB_LIGHTS_PER_CELL + 1);
        if (len != ctx->B.lightsLen) {
            std::vector<float> rec(ctx->hostLights.begin(), ctx->hostLights.begin() + SB_MAX_LIGHTS * SB_LIGHT_STRIDE);
            s = sb_upload_lights(ctx, rec.data(), ctx->lightCount, ctx->emitterBase, ctx->emitterCount, 1);
            if (s != SB_OK) return s;
        }
        ctx->lightGridDirty = true;
    }
    return SB_OK;
}

sb_status sb_solve(sb_ctx* ctx, uint32_t ci, uint32_t probeOffset, uint32_t updatedCount) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
        return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", ci);
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    if (ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "TLAS not built (sb_build_tlas)");
    if (!ctx->B.lights) return fail(ctx, SB_ERR_NOT_READY, "no lights uploaded (sb_upload_lights, count may be 0)");
    Cascade& K = ctx->casc[ci];
    if (updatedCount > K.probeTotal) updatedCount = K.probeTotal;
    probeOffset %= K.probeTotal;
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    s = light_grid_if_needed(ctx);
    if (s != SB_OK) return s;
    s = flat_if_needed(ctx);
    if (s != SB_OK) return s;
    DevScene S = dev_scene(ctx);
    DevCascade D = dev_cascade(ctx, ci, probeOffset, updatedCount);
    DevParams P;
    std::memcpy(&P, &ctx->params, sizeof P);
    // shadow-job queue: up to one job per (ray, light); solves larger than the
    // queue cap run as several probe-slot chunks before the blend
    const uint64_t perProbe = (uint64_t)K.grid.raysPerProbe * (ctx->lightCount ? ctx->lightCount : 1u);
    uint64_t want = perProbe * updatedCount;
    if (want > kJobCapMax) want = kJobCapMax - kJobCapMax % perProbe;
    if (want < perProbe) want = perProbe;
    if (want > ctx->jobCap) {
        release(ctx->jobs);
        size_t c = 0;
        CK(grow(ctx->jobs, c, (size_t)want * 2));
        ctx->jobCap = (uint32_t)want;
    }
    const uint32_t chunk = (uint32_t)(ctx->jobCap / perProbe);
    const bool fullSolve = probeOffset == 0 && updatedCount == K.probeTotal && updatedCount <= chunk;
    if (ctx->tune.sortKey >= 2 && fullSolve) D.issueOrder = K.tileOrder;  // every probe in one chunk: tile by tile
    // (the refill form on the 8-wide tree has no fixed batches to order)
    const bool costOrder = ctx->tune.sortKey == 3 && fullSolve && !(SB_PRIMARY_REFILL && S.wideNodes);
    if (costOrder) {  // this solve records its batch costs and orders the next one by them
        D.batchCost = K.batchCost;
        D.batchOrder = K.batchOrderReady ? K.batchOrder : nullptr;
        D.batchOrderOut = K.batchOrder;
    }
    if (ctx->countersOn) CK(cudaMemsetAsync(ctx->dCounters, 0, 128, ctx->stream));
    const bool timing = !ctx->capturing;  // events inside a capture would not be re-recorded by replays
    if (timing) CK(cudaEventRecord(ctx->ev0, ctx->stream));
    ctx->singleChunk = updatedCount <= chunk;
    for (uint32_t s0 = 0; s0 < updatedCount; s0 += chunk) {
        uint32_t n = updatedCount - s0 < chunk ? updatedCount - s0 : chunk;
        CK(launch_trace(S, D, P, ctx->dErr, ctx->countersOn ? ctx->dCounters : nullptr, ctx->dWork, ctx->tune,
                        ctx->stream, ctx->jobs, ctx->jobCap, s0, n, timing ? ctx->evA : nullptr,
                        timing ? ctx->evB : nullptr, timing ? ctx->evC : nullptr));
    }
    if (ctx->emitterCount) CK(launch_emitter_vis(S, D, P, ctx->dErr, ctx->stream));
    if (timing) CK(cudaEventRecord(ctx->evMid, ctx->stream));
    CK(launch_blend_upload(D, P, ctx->stream));
    if (K.reflTier >= SB_REFLECT_HIGH) {
        // glossyKernel after the blend (gi_probes.js:3829-3835): this solve resolves
        // the texels of phase D.glossyPhase, the next one the following phase
        CK(launch_glossy(D, P, ctx->stream));
        K.glossyPhase = (K.glossyPhase + 1u) % K.glossyInterval;
    }
    if (costOrder) K.batchOrderReady = true;
    if (timing) CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->timed = ctx->timed || timing;
    if (timing) ctx->lastWasGraph = false;
    return SB_OK;
}

// Host-side preparation a solve of cascade ci needs (validation, derived
// layouts, light grid, scene BVH and its marks): done before any enqueue.
static sb_status solve_prepare(sb_ctx* ctx, uint32_t ci) {
    if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
        return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", ci);
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    if (ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "TLAS not built (sb_build_tlas)");
    if (!ctx->B.lights) return fail(ctx, SB_ERR_NOT_READY, "no lights uploaded (sb_upload_lights, count may be 0)");
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s == SB_OK) s = light_grid_if_needed(ctx);
    if (s == SB_OK) s = flat_if_needed(ctx);
    return s;
}

static cudaError_t ensure_sync_event(sb_ctx* c) {
    return c->syncEv ? cudaSuccess : cudaEventCreateWithFlags(&c->syncEv, cudaEventDisableTiming);
}

// The kernel arguments of a batch from the items' current state (scenes,
// cascades, parameters); grows the lead context's job queue when allowed.
static sb_status build_batch(const sb_solve_item* items, uint32_t count, BatchArgs& B, bool mayGrow) {
    sb_ctx* lead = items[0].ctx;
    sb_ctx* ctx = lead;  // error reporting (CK)
    std::memset(&B, 0, sizeof B);
    uint64_t rayBase = 0, jobs = 0;
    uint32_t blend = 0;
    for (uint32_t i = 0; i < count; ++i) {
        sb_ctx* c = items[i].ctx;
        // emitters or reflection lobes set after a capture: the batched kernels cover neither
        if (c->emitterCount || c->reflectTier)
            return fail(lead, SB_ERR_UNSUPPORTED, "item %u: emitters / reflection lobes are solved by sb_solve only", i);
        const uint32_t ci = items[i].cascade;
        Cascade& K = c->casc[ci];
        const uint32_t cnt = items[i].updatedCount > K.probeTotal ? K.probeTotal : items[i].updatedCount;
        BatchItem& I = B.it[i];
        I.W.S = dev_scene(c);
        I.W.C = dev_cascade(c, ci, items[i].probeOffset % K.probeTotal, cnt);
        std::memcpy(&I.W.P, &c->params, sizeof I.W.P);
        I.W.err = c->dErr;
        I.W.counters = nullptr;
        I.W.work = lead->dWork;
        I.W.slotBegin = 0;
        I.W.slotCount = cnt;
        I.W.smemTlas = 0;
        I.W.order = lead->tune.sortKey == 1 ? 0u : 1u;
        if (lead->tune.sortKey >= 2 && I.W.C.probeOffset == 0 && cnt == K.probeTotal) I.W.C.issueOrder = K.tileOrder;
        const uint64_t rays = (uint64_t)cnt * K.grid.raysPerProbe;
        I.rayBase = (uint32_t)rayBase;
        I.rays = (uint32_t)rays;
        rayBase = (rayBase + rays + 31) & ~31ull;
        I.blendBase = blend;
        I.blendBlocks = blend_blocks(cnt);
        blend += I.blendBlocks;
        jobs += rays * (c->lightCount ? c->lightCount : 1u);
    }
    if (rayBase >= (1ull << 26))
        return fail(lead, SB_ERR_INVALID_ARG, "batch of %llu rays exceeds the 2^26 job tag range",
                    (unsigned long long)rayBase);
    if (jobs > kJobCapMax)
        return fail(lead, SB_ERR_UNSUPPORTED, "batch needs %llu shadow-job slots (max %llu): split it",
                    (unsigned long long)jobs, (unsigned long long)kJobCapMax);
    if (jobs > lead->jobCap) {
        if (!mayGrow) return fail(lead, SB_ERR_NOT_READY, "the batch's job queue must grow outside a graph");
        release(lead->jobs);
        size_t c = 0;
        CK(grow(lead->jobs, c, (size_t)jobs * 2));
        lead->jobCap = (uint32_t)jobs;
    }
    for (uint32_t i = 0; i < count; ++i) {
        B.it[i].W.jobs = lead->jobs;
        B.it[i].W.jobCap = lead->jobCap;
    }
    B.n = count;
    B.totalRays = (uint32_t)rayBase;
    B.blendBlocks = blend;
    B.work = lead->dWork;
    B.counters = lead->countersOn ? lead->dCounters : nullptr;
    return SB_OK;
}

// Cross-context ordering around work on the lead's stream: `before` makes the
// lead wait for the other contexts' pending work, else the others wait for
// the lead's.
static sb_status join_streams(const sb_solve_item* items, uint32_t count, bool before) {
    sb_ctx* lead = items[0].ctx;
    sb_ctx* ctx = lead;
    bool recorded = false;
    for (uint32_t i = 1; i < count; ++i) {
        sb_ctx* c = items[i].ctx;
        if (c->stream == lead->stream) continue;
        if (before) {
            CK(ensure_sync_event(c));
            CK(cudaEventRecord(c->syncEv, c->stream));
            CK(cudaStreamWaitEvent(lead->stream, c->syncEv, 0));
        } else {
            CK(ensure_sync_event(lead));
            if (!recorded) CK(cudaEventRecord(lead->syncEv, lead->stream));
            recorded = true;
            CK(cudaStreamWaitEvent(c->stream, lead->syncEv, 0));
        }
    }
    return SB_OK;
}

// One launch per stage over every item (sb_solve_batch); the items' contexts
// share a device, and the first item's context owns the ray queue, the job
// queue and the stream the batch runs on.
static sb_status enqueue_batch(const sb_solve_item* items, uint32_t count) {
    sb_ctx* lead = items[0].ctx;
    sb_ctx* ctx = lead;  // error reporting (CK)
    static thread_local BatchArgs B;
    sb_status s = build_batch(items, count, B, !lead->capturing);
    if (s != SB_OK) return s;
    // inside a capture the graph's launch does the joins
    if (!lead->capturing && (s = join_streams(items, count, true)) != SB_OK) return s;
    const bool timing = !lead->capturing;
    if (B.counters) CK(cudaMemsetAsync(lead->dCounters, 0, 128, lead->stream));
    if (timing) CK(cudaEventRecord(lead->ev0, lead->stream));
    CK(launch_trace_batch(B, lead->tune, lead->stream, timing ? lead->evA : nullptr, timing ? lead->evB : nullptr,
                          timing ? lead->evC : nullptr));
    if (timing) CK(cudaEventRecord(lead->evMid, lead->stream));
    CK(launch_blend_upload_batch(B, lead->stream));
    if (timing) {
        CK(cudaEventRecord(lead->ev1, lead->stream));
        lead->timed = true;
        lead->singleChunk = true;
        lead->lastWasGraph = false;
    }
    if (!lead->capturing) return join_streams(items, count, false);
    return SB_OK;
}

static sb_status check_batch(const sb_solve_item* items, uint32_t count) {
    if (!items || count == 0 || !items[0].ctx) return SB_ERR_INVALID_ARG;
    sb_ctx* lead = items[0].ctx;
    if (count > SB_BATCH_MAX) return fail(lead, SB_ERR_INVALID_ARG, "%u items > %u per batch", count, SB_BATCH_MAX);
    for (uint32_t i = 0; i < count; ++i) {
        sb_ctx* c = items[i].ctx;
        if (!c || c->device != lead->device) return fail(lead, SB_ERR_INVALID_ARG, "item %u: null context or another device", i);
        if (c->emitterCount)
            return fail(lead, SB_ERR_UNSUPPORTED, "item %u: giEmitter records are solved by sb_solve only", i);
        if (c->reflectTier)
            return fail(lead, SB_ERR_UNSUPPORTED, "item %u: reflection lobes are solved by sb_solve only", i);
        for (uint32_t j = 0; j < i; ++j)
            if (items[j].ctx == c && items[j].cascade == items[i].cascade)
                return fail(lead, SB_ERR_INVALID_ARG, "items %u and %u solve the same cascade", j, i);
        sb_status s = solve_prepare(c, items[i].cascade);
        if (s != SB_OK) {
            if (c != lead) lead->err = "item " + std::to_string(i) + ": " + c->err;
            return s;
        }
    }
    return SB_OK;
}

sb_status sb_solve_batch(const sb_solve_item* items, uint32_t count) {
    sb_status s = check_batch(items, count);
    if (s != SB_OK) return s;
    cudaSetDevice(items[0].ctx->device);
    return enqueue_batch(items, count);
}

// ---------------------------------------------------------------- graphs

static void graph_release(sb_ctx* ctx) {
    auto& G = ctx->graph;
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.graph) cudaGraphDestroy(G.graph);
    G.exec = nullptr;
    G.graph = nullptr;
    for (auto& n : G.nodes) n = nullptr;
    G.lanes.clear();
    G.items.clear();
    G.keys.clear();
}

static void graph_free_streams(sb_ctx* ctx) {
    auto& G = ctx->graph;
    for (cudaStream_t s : G.branches) cudaStreamDestroy(s);
    for (cudaEvent_t e : G.joins) cudaEventDestroy(e);
    if (G.fork) cudaEventDestroy(G.fork);
    G.branches.clear();
    G.joins.clear();
    G.fork = nullptr;
}

// Every context a frame touches, once.
static std::vector<sb_ctx*> frame_contexts(const std::vector<sb_ctx::Graph::Lane>& lanes,
                                           const std::vector<sb_solve_item>& items) {
    std::vector<sb_ctx*> out;
    auto add = [&](sb_ctx* c) {
        for (sb_ctx* o : out)
            if (o == c) return;
        out.push_back(c);
    };
    for (const auto& it : items) add(it.ctx);
    for (const auto& l : lanes) add(l.ctx);
    return out;
}

static sb_status run_lane(const sb_ctx::Graph::Lane& l) {
    for (size_t r = 0; r < l.roots.size(); ++r) {
        sb_status s = sb_refit_blas(l.ctx, l.roots[r], l.ends[r]);
        if (s != SB_OK) return s;
    }
    return l.refitTlas ? sb_update_transforms(l.ctx, nullptr, nullptr, 0) : SB_OK;
}

// Runs the frame once as ordinary launches (it applies the host-side effects:
// packs, refit layout checks, moved-slot marks, queue growth), then captures
// it: each lane a branch forked from the owner's stream, joined ahead of the
// batched solve. The batched kernels' nodes are kept so replays refresh their
// parameters.
static sb_status graph_capture(sb_ctx* lead, std::vector<sb_ctx::Graph::Lane> lanes,
                               std::vector<sb_solve_item> items) {
    sb_ctx* ctx = lead;
    const std::vector<sb_ctx*> all = frame_contexts(lanes, items);
    for (const auto& l : lanes) {
        sb_status s = run_lane(l);
        if (s != SB_OK) return s;
    }
    sb_status s = sb_solve_batch(items.data(), (uint32_t)items.size());
    if (s != SB_OK) return s;
    for (sb_ctx* c : all)
        if ((s = sb_synchronize(c)) != SB_OK) return s;
    graph_release(lead);
    auto& G = lead->graph;
    while (G.branches.size() < lanes.size()) {
        cudaStream_t st;
        cudaEvent_t ev;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        G.branches.push_back(st);
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        G.joins.push_back(ev);
    }
    if (!G.fork) CK(cudaEventCreateWithFlags(&G.fork, cudaEventDisableTiming));
    for (sb_ctx* c : all) c->capturing = true;
    cudaError_t e = cudaStreamBeginCapture(lead->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(G.fork, lead->stream);
    for (size_t i = 0; i < lanes.size() && e == cudaSuccess && s == SB_OK; ++i) {
        sb_ctx* c = lanes[i].ctx;
        e = cudaStreamWaitEvent(G.branches[i], G.fork, 0);
        if (e != cudaSuccess) break;
        cudaStream_t saved = c->stream;
        c->stream = G.branches[i];
        s = run_lane(lanes[i]);
        c->stream = saved;
        if (s == SB_OK) e = cudaEventRecord(G.joins[i], G.branches[i]);
        if (e == cudaSuccess && s == SB_OK) e = cudaStreamWaitEvent(lead->stream, G.joins[i], 0);
    }
    if (e == cudaSuccess && s == SB_OK) s = enqueue_batch(items.data(), (uint32_t)items.size());
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(lead->stream, &graph);
    for (sb_ctx* c : all) c->capturing = false;
    if (e == cudaSuccess) e = e2;
    if (s != SB_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (s != SB_OK) return s;
        CK(e);
    }
    G.graph = graph;
    size_t n = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    CK(cudaGraphGetNodes(graph, nodes.data(), &n));
    // stages without a kernel of their own (null) are done inside another one
    const void* fn[5] = {trace_batch_kernel(0), trace_batch_kernel(1), trace_batch_kernel(2), trace_batch_kernel(3),
                         blend_batch_kernel()};
    int found = 0, expected = 0;
    for (const void* f : fn) expected += f ? 1 : 0;
    G.kernelNodes = 0;
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType t;
        CK(cudaGraphNodeGetType(node, &t));
        if (t != cudaGraphNodeTypeKernel) continue;
        ++G.kernelNodes;
        cudaKernelNodeParams p;
        CK(cudaGraphKernelNodeGetParams(node, &p));
        for (int k = 0; k < 5; ++k)
            if (fn[k] && p.func == fn[k]) {
                G.nodes[k] = node;
                G.params[k] = p;
                ++found;
            }
    }
    if (found != expected) {
        graph_release(lead);
        return fail(lead, SB_ERR_CUDA, "captured frame holds %d of the %d batched kernels", found, expected);
    }
    CK(cudaGraphInstantiate(&G.exec, graph, 0));
    G.lanes = std::move(lanes);
    G.items = std::move(items);
    for (sb_ctx* c : all) G.keys.push_back({c, {c->structGen, c->packEpoch}});
    return SB_OK;
}

static sb_status graph_launch(sb_ctx* lead) {
    sb_ctx* ctx = lead;
    auto& G = lead->graph;
    if (!G.exec) return fail(lead, SB_ERR_NOT_READY, "no captured frame (sb_graph_capture_frame / _batch)");
    for (const auto& k : G.keys)
        if (k.first->structGen != k.second.first || k.first->packEpoch != k.second.second) {
            // buffers or layouts changed since the capture: this frame runs as
            // ordinary launches and is captured again for the next replays
            auto lanes = G.lanes;
            auto items = G.items;
            return graph_capture(lead, std::move(lanes), std::move(items));
        }
    const uint32_t count = (uint32_t)G.items.size();
    for (const auto& it : G.items) {
        sb_status s = solve_prepare(it.ctx, it.cascade);
        if (s != SB_OK) return s;
    }
    static thread_local BatchArgs B;
    sb_status s = build_batch(G.items.data(), count, B, false);
    if (s != SB_OK) return s;
    void* args[1] = {&B};
    for (int k = 0; k < 5; ++k) {
        if (!G.nodes[k]) continue;
        cudaKernelNodeParams p = G.params[k];
        p.kernelParams = args;
        p.extra = nullptr;
        CK(cudaGraphExecKernelNodeSetParams(G.exec, G.nodes[k], &p));
    }
    const std::vector<sb_ctx*> all = frame_contexts(G.lanes, G.items);
    for (sb_ctx* c : all) {
        if (c == lead || c->stream == lead->stream) continue;
        CK(ensure_sync_event(c));
        CK(cudaEventRecord(c->syncEv, c->stream));
        CK(cudaStreamWaitEvent(lead->stream, c->syncEv, 0));
    }
    CK(cudaEventRecord(lead->ev0, lead->stream));
    CK(cudaGraphLaunch(G.exec, lead->stream));
    for (uint32_t k = 0; k < G.kernelNodes; ++k) note_launch();
    CK(cudaEventRecord(lead->ev1, lead->stream));
    G.timed = true;
    lead->timed = true;
    lead->lastWasGraph = true;
    CK(ensure_sync_event(lead));
    CK(cudaEventRecord(lead->syncEv, lead->stream));
    for (sb_ctx* c : all)
        if (c != lead && c->stream != lead->stream) CK(cudaStreamWaitEvent(c->stream, lead->syncEv, 0));
    return SB_OK;
}

sb_status sb_graph_capture_batch(const sb_frame_lane* lanes, uint32_t laneCount, const sb_solve_item* items,
                                 uint32_t itemCount) {
    if (!items || itemCount == 0 || !items[0].ctx || (laneCount && !lanes)) return SB_ERR_INVALID_ARG;
    sb_ctx* lead = items[0].ctx;
    if (laneCount > 64) return fail(lead, SB_ERR_INVALID_ARG, "%u lanes > 64", laneCount);
    std::vector<sb_ctx::Graph::Lane> L;
    for (uint32_t i = 0; i < laneCount; ++i) {
        const sb_frame_lane& l = lanes[i];
        if (!l.ctx || l.ctx->device != lead->device || (l.refitCount && (!l.refitRoots || !l.refitEnds)))
            return fail(lead, SB_ERR_INVALID_ARG, "lane %u: bad context or refit ranges", i);
        for (uint32_t j = 0; j < i; ++j)
            if (lanes[j].ctx == l.ctx) return fail(lead, SB_ERR_INVALID_ARG, "lanes %u and %u share a context", j, i);
        sb_ctx::Graph::Lane x{l.ctx, {}, {}, l.refitTlas};
        x.roots.assign(l.refitRoots, l.refitRoots + l.refitCount);
        x.ends.assign(l.refitEnds, l.refitEnds + l.refitCount);
        L.push_back(std::move(x));
    }
    sb_status s = check_batch(items, itemCount);
    if (s != SB_OK) return s;
    cudaSetDevice(lead->device);
    return graph_capture(lead, std::move(L), std::vector<sb_solve_item>(items, items + itemCount));
}

sb_status sb_graph_capture_frame(sb_ctx* ctx, uint32_t cascade, uint32_t probeOffset, uint32_t updatedCount,
                                 const uint32_t* refitRoots, const uint32_t* refitEnds, uint32_t refitCount,
                                 int32_t refitTlas) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    sb_frame_lane lane{ctx, refitRoots, refitEnds, refitCount, refitTlas};
    sb_solve_item item{ctx, cascade, probeOffset, updatedCount};
    const bool anyLane = refitCount > 0 || refitTlas;
    return sb_graph_capture_batch(anyLane ? &lane : nullptr, anyLane ? 1u : 0u, &item, 1);
}

sb_status sb_graph_launch(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    return graph_launch(ctx);
}

// ---------------------------------------------------------------- autotuner

// A copy of one cascade's probe state (histories, atlases), so trial solves
// leave it as they found it.
struct CascadeSnapshot {
    sb_ctx* ctx = nullptr;
    uint32_t ci = 0;
    uint32_t glossyPhase = 0;
    struct Region { void* live; void* copy; size_t bytes; };
    std::vector<Region> regions;  // histories, atlases, emitter visibility, reflection lobes
    CascadeSnapshot() = default;
    CascadeSnapshot(const CascadeSnapshot&) = delete;
    CascadeSnapshot& operator=(const CascadeSnapshot&) = delete;

    cudaError_t copy(bool save) {
        for (auto& r : regions) {
            cudaError_t e = cudaMemcpyAsync(save ? r.copy : r.live, save ? r.live : r.copy, r.bytes,
                                            cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    cudaError_t save(sb_ctx* c, uint32_t cascade) {
        ctx = c;
        ci = cascade;
        Cascade& K = c->casc[cascade];
        glossyPhase = K.glossyPhase;
        const size_t hist = (size_t)K.probeTotal * 64, texels = (size_t)K.atlasW * K.atlasH;
        const size_t gt = (size_t)K.probeTotal * K.glossyTile * K.glossyTile;
        const size_t ga = (size_t)K.glossyTilesX * K.glossyTile * K.glossyTilesY * K.glossyTile;
        const Region want[] = {{K.irr, nullptr, hist * 16}, {K.depth, nullptr, hist * 8},
                               {K.atlas, nullptr, texels * 8}, {K.depthAtlas, nullptr, texels * 8},
                               {K.emitterVis, nullptr, (size_t)K.probeTotal * EMITTER_CAP * 4},
                               {K.roughSpec, nullptr, hist * 16}, {K.roughAtlas, nullptr, texels * 8},
                               {K.glossyNum, nullptr, gt * 16}, {K.glossyDen, nullptr, gt * 4},
                               {K.glossyAtlas, nullptr, ga * 8}};
        for (const Region& r : want) {
            if (!r.live || !r.bytes) continue;
            Region x = r;
            cudaError_t e = cudaMalloc(&x.copy, x.bytes);
            if (e != cudaSuccess) return e;
            regions.push_back(x);
        }
        return copy(true);
    }
    cudaError_t restore() {
        ctx->casc[ci].glossyPhase = glossyPhase;
        cudaError_t e = copy(false);
        return e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
    }
    ~CascadeSnapshot() {
        for (auto& r : regions) release(r.copy);
    }
};

// Minimum device time (lead->ev0 .. ev1) of `reps` runs after one warm-up.
static sb_status time_min(sb_ctx* lead, const std::vector<sb_ctx*>& all, const std::function<sb_status()>& run,
                          int reps, float& best) {
    best = 3.4e38f;
    for (int rep = 0; rep <= reps; ++rep) {
        sb_status s = run();
        for (sb_ctx* c : all)
            if (s == SB_OK) s = sb_synchronize(c);
        if (s != SB_OK) return s;
        float m = 0.0f;
        if (rep > 0 && cudaEventElapsedTime(&m, lead->ev0, lead->ev1) == cudaSuccess && m < best) best = m;
    }
    return SB_OK;
}

// Times full solves of cascade ci under each candidate tuning and keeps the
// fastest. Candidates: the scene BVH kinds (8-wide / binary / the reference's
// two-level walk), traversal block sizes 128 / 192 / 256, the four ray issue
// orders (sortKey 0-3), for the 8-wide tree 0 / 73 / 512 top nodes staged in
// shared memory, and for the two-level walk TLAS staging in shared memory off /
// up to 512 nodes. The cascade's histories and atlases are restored afterwards, so
// tuning leaves the probe state as it found it.
sb_status sb_autotune(sb_ctx* ctx, uint32_t ci, sb_tuning* chosen) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    sb_status s = solve_prepare(ctx, ci);
    if (s != SB_OK) return s;
    const uint32_t probes = ctx->casc[ci].probeTotal;
    CascadeSnapshot snap;
    CK(snap.save(ctx, ci));
    const sb_tuning saved{ctx->tune.block, ctx->tune.sortKey, ctx->tune.smemTlasNodes, ctx->bvhKind,
                          ctx->tune.smemWideNodes};
    const bool savedCounters = ctx->countersOn;
    ctx->countersOn = false;
    sb_tuning best = saved;
    float bestMs = 3.4e38f;
    const uint32_t kinds[3] = {1u, 2u, 0u}, blocks[3] = {128u, 192u, 256u};
    const uint32_t wideDepth[3] = {0u, 73u, 512u};  // none, the top three levels, 512 nodes
    // shared-memory staging: the TLAS for the two-level walk, the top 8-wide nodes for kind 1
    for (uint32_t kind : kinds)
        for (uint32_t block : blocks)
            for (uint32_t sort = 0; sort < 4 && s == SB_OK; ++sort)
                for (uint32_t sm = 0; sm < (kind == 0 ? 2u : kind == 1 ? 3u : 1u) && s == SB_OK; ++sm) {
                    sb_tuning t{block, sort, kind == 0 ? (sm ? 512u : 0u) : saved.smemTlasNodes, kind,
                                kind == 1 ? wideDepth[sm] : 0u};
                    if ((s = sb_set_tuning(ctx, &t)) != SB_OK) break;
                    float ms = 0.0f;
                    s = time_min(ctx, {ctx}, [&] { return sb_solve(ctx, ci, 0, probes); }, 3, ms);
                    if (s == SB_OK && ms < bestMs) {
                        bestMs = ms;
                        best = t;
                    }
                }
    cudaError_t e = snap.restore();
    ctx->countersOn = savedCounters;
    sb_status s2 = sb_set_tuning(ctx, s == SB_OK && e == cudaSuccess ? &best : &saved);
    if (s != SB_OK) return s;
    CK(e);
    if (s2 != SB_OK) return s2;
    if (chosen) *chosen = best;
    return SB_OK;
}

// The batch's launch parameters (the lead context's block size and ray issue
// order) timed on the batched solve itself; each context keeps its own scene
// BVH kind. Every item's probe state is restored afterwards.
sb_status sb_autotune_batch(const sb_solve_item* items, uint32_t count, sb_tuning* chosen) {
    sb_status s = check_batch(items, count);
    if (s != SB_OK) return s;
    sb_ctx* lead = items[0].ctx;
    sb_ctx* ctx = lead;
    cudaSetDevice(lead->device);
    std::vector<CascadeSnapshot> snaps(count);
    std::vector<sb_ctx*> all;
    for (uint32_t i = 0; i < count; ++i) {
        CK(snaps[i].save(items[i].ctx, items[i].cascade));
        bool seen = false;
        for (sb_ctx* c : all) seen = seen || c == items[i].ctx;
        if (!seen) all.push_back(items[i].ctx);
    }
    const sb_tuning saved{lead->tune.block, lead->tune.sortKey, lead->tune.smemTlasNodes, lead->bvhKind,
                          lead->tune.smemWideNodes};
    sb_tuning best = saved;
    float bestMs = 3.4e38f;
    const uint32_t blocks[3] = {128u, 192u, 256u};
    for (uint32_t block : blocks)
        for (uint32_t sort = 0; sort < 3 && s == SB_OK; ++sort) {
            sb_tuning t{block, sort, saved.smemTlasNodes, saved.bvhKind, saved.smemWideNodes};
            if ((s = sb_set_tuning(lead, &t)) != SB_OK) break;
            float ms = 0.0f;
            s = time_min(lead, all, [&] { return sb_solve_batch(items, count); }, 3, ms);
            if (s == SB_OK && ms < bestMs) {
                bestMs = ms;
                best = t;
            }
        }
    cudaError_t e = cudaSuccess;
    for (auto& sn : snaps)
        if (e == cudaSuccess) e = sn.restore();
    sb_status s2 = sb_set_tuning(lead, s == SB_OK && e == cudaSuccess ? &best : &saved);
    if (s != SB_OK) return s;
    CK(e);
    if (s2 != SB_OK) return s2;
    if (chosen) *chosen = best;
    return SB_OK;
}

sb_status sb_graph_destroy(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    graph_release(ctx);
    graph_free_streams(ctx);
    return SB_OK;
}

// ---------------------------------------------------------------- adjoint

sb_status sb_forward_record(sb_ctx* ctx, uint32_t ci, uint32_t solves, const float* target, double* loss) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    if (solves < 1 || solves > 8) return fail(ctx, SB_ERR_INVALID_ARG, "solves=%u outside [1,8]", solves);
    if (target && !loss) return fail(ctx, SB_ERR_INVALID_ARG, "loss is null");
    if (ci >= SB_MAX_CASCADES || !ctx->casc[ci].configured)
        return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", ci);
    if (ctx->emitterCount)
        return fail(ctx, SB_ERR_UNSUPPORTED, "the adjoint does not cover giEmitter virtual rays");
    if (ctx->reflectTier)
        return fail(ctx, SB_ERR_UNSUPPORTED, "the adjoint does not cover the reflection lobes");
    cudaSetDevice(ctx->device);
    Cascade& K = ctx->casc[ci];
    auto& T = ctx->tape;
    T.ready = false;
    const uint32_t probes = K.probeTotal, rays = K.grid.raysPerProbe;
    const size_t nRay = (size_t)probes * rays, texels = (size_t)K.atlasW * K.atlasH;
    CK(grow(T.hits, T.hitsCap, solves * nRay));
    CK(grow(T.vis, T.visCap, solves * nRay));
    CK(grow(T.hist, T.histCap, (solves + 1) * (size_t)probes * 64));
    CK(grow(T.atlas, T.atlasCap, solves * texels));
    CK(grow(T.E, T.ECap, (size_t)probes * 36));
    CK(grow(T.loss, T.lossCap, 1));
    if (!T.evF0) {
        for (cudaEvent_t* e : {&T.evF0, &T.evF1, &T.evB0, &T.evB1}) CK(cudaEventCreate(e));
    }
    CK(cudaEventRecord(T.evF0, ctx->stream));
    CK(launch_clear_cascade(dev_cascade(ctx, ci, 0, 0), ctx->stream));
    const size_t histBytes = (size_t)probes * 64 * sizeof(float4), atlasBytes = texels * sizeof(uint2);
    for (uint32_t s = 0; s < solves; ++s) {
        CK(cudaMemcpyAsync(T.hist + s * (size_t)probes * 64, K.irr, histBytes, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(T.atlas + s * texels, K.atlas, atlasBytes, cudaMemcpyDeviceToDevice, ctx->stream));
        ctx->recordE = s + 1 == solves ? T.E : nullptr;
        sb_status st = sb_solve(ctx, ci, 0, probes);
        ctx->recordE = nullptr;
        if (st != SB_OK) return st;
        CK(cudaMemcpyAsync(T.hits + s * nRay, K.hits, nRay * sizeof(uint4), cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(T.vis + s * nRay, K.vis, nRay * sizeof(uint4), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CK(cudaMemcpyAsync(T.hist + solves * (size_t)probes * 64, K.irr, histBytes, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    T.hasTarget = target != nullptr;
    if (target) {
        CK(grow(T.target, T.targetCap, (size_t)probes * 36 * 3));
        CK(grow(T.gE, T.gECap, (size_t)probes * 36));
        CK(cudaMemcpyAsync(T.target, target, (size_t)probes * 36 * 3 * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(launch_adjoint_loss(T.E, T.target, probes * 36, T.gE, T.loss, ctx->stream));
    }
    CK(cudaEventRecord(T.evF1, ctx->stream));
    T.timedF = true;
    T.cascade = ci;
    T.solves = solves;
    T.probes = probes;
    T.rays = rays;
    T.texels = (uint32_t)texels;
    T.epoch = ctx->epoch;
    T.ready = true;
    if (target) {
        CK(cudaMemcpyAsync(loss, T.loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        return sb_synchronize(ctx);
    }
    return SB_OK;
}

sb_status sb_backward(sb_ctx* ctx, sb_grads* grads) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    auto& T = ctx->tape;
    if (!T.ready || !T.hasTarget) return fail(ctx, SB_ERR_NOT_READY, "no recorded forward with a target");
    if (T.epoch != ctx->epoch)
        return fail(ctx, SB_ERR_NOT_READY, "scene, lights, parameters or cascade changed since sb_forward_record");
    cudaSetDevice(ctx->device);
    const uint32_t probes = T.probes, mc = ctx->B.materialCount, lc = ctx->lightCount;
    const size_t nRay = (size_t)probes * T.rays, hist = (size_t)probes * 64;
    const size_t nParam = 6 * (size_t)mc + lc;
    CK(grow(T.shaded, T.shadedCap, nRay));
    CK(grow(T.gR, T.gRCap, nRay));
    CK(grow(T.gH, T.gHCap, 2 * hist));
    CK(grow(T.gA, T.gACap, 2 * (size_t)T.texels));
    CK(grow(T.gParam, T.gParamCap, nParam ? nParam : 1));
    CK(cudaEventRecord(T.evB0, ctx->stream));
    CK(cudaMemsetAsync(T.gParam, 0, nParam * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(T.gH, 0, hist * sizeof(float4), ctx->stream));
    const DevScene S = dev_scene(ctx);
    DevParams P;
    std::memcpy(&P, &ctx->params, sizeof P);
    float4* gHnext = T.gH;              // dL/dH after solve s (from solve s + 1's blend)
    const float4* gAnext = nullptr;     // dL/dAtlas written by solve s (read by solve s + 1)
    for (int s = (int)T.solves - 1; s >= 0; --s) {
        DevCascade D = dev_cascade(ctx, T.cascade, 0, probes);
        D.hits = T.hits + s * nRay;
        D.vis = T.vis + s * nRay;
        D.atlasPrev = T.atlas + (size_t)s * T.texels;
        D.rayData = T.shaded;
        D.eOut = nullptr;
        const float4* Hs = T.hist + (size_t)s * hist;
        const float4* Hs1 = T.hist + (size_t)(s + 1) * hist;
        const bool last = s + 1 == (int)T.solves;
        CK(launch_upload_bwd(D, P, Hs1, last ? T.gE : nullptr, gAnext, gHnext, ctx->stream));
        float4* gAcur = T.gA + (size_t)(s & 1) * T.texels;
        float4* gHprev = gHnext == T.gH ? T.gH + hist : T.gH;
        CK(cudaMemsetAsync(gAcur, 0, (size_t)T.texels * sizeof(float4), ctx->stream));
        CK(launch_shade(S, D, P, probes, ctx->stream));
        CK(launch_blend_bwd(D, P, T.shaded, Hs, gHnext, gHprev, T.gR, ctx->stream));
        CK(launch_shade_bwd(S, D, P, T.gR, T.gParam, gAcur, ctx->stream));
        gHnext = gHprev;
        gAnext = gAcur;
    }
    CK(cudaEventRecord(T.evB1, ctx->stream));
    T.timedB = true;
    std::vector<double> g(nParam);
    if (nParam) CK(cudaMemcpyAsync(g.data(), T.gParam, nParam * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sb_status st = sb_synchronize(ctx);
    if (st != SB_OK) return st;
    if (grads) {
        for (uint32_t i = 0; i < 3 * mc; ++i) {
            if (grads->dAlbedo) grads->dAlbedo[i] = (float)g[i];
            if (grads->dEmissive) grads->dEmissive[i] = (float)g[3 * (size_t)mc + i];
        }
        if (grads->dIntensity)
            for (uint32_t l = 0; l < lc; ++l) grads->dIntensity[l] = (float)g[6 * (size_t)mc + l];
    }
    return SB_OK;
}

sb_status sb_raycast(sb_ctx* ctx, const float* ro, const float* rd, uint32_t n, float* tOut, int32_t* triOut,
                     int32_t* instOut) {
    if (!ctx || (n && (!ro || !rd || !tOut || !triOut || !instOut))) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!ctx->sceneLoaded || ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "scene / TLAS not ready");
    if (n == 0) return SB_OK;
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    s = flat_if_needed(ctx);
    if (s != SB_OK) return s;
    float *dro = nullptr, *drd = nullptr, *dt = nullptr;
    int32_t *dtri = nullptr, *dinst = nullptr;
    CK(cudaMallocAsync(&dro, (size_t)n * 12, ctx->stream));
    CK(cudaMallocAsync(&drd, (size_t)n * 12, ctx->stream));
    CK(cudaMallocAsync(&dt, (size_t)n * 4, ctx->stream));
    CK(cudaMallocAsync(&dtri, (size_t)n * 4, ctx->stream));
    CK(cudaMallocAsync(&dinst, (size_t)n * 4, ctx->stream));
    CK(cudaMemcpyAsync(dro, ro, (size_t)n * 12, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(drd, rd, (size_t)n * 12, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_raycast(dev_scene(ctx), dro, drd, n, dt, dtri, dinst, ctx->dErr, ctx->stream));
    CK(cudaMemcpyAsync(tOut, dt, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(triOut, dtri, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(instOut, dinst, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    cudaFreeAsync(dro, ctx->stream); cudaFreeAsync(drd, ctx->stream); cudaFreeAsync(dt, ctx->stream);
    cudaFreeAsync(dtri, ctx->stream); cudaFreeAsync(dinst, ctx->stream);
    return sb_synchronize(ctx);
}

// The traversal queries on the caller's device arrays, enqueued on the
// context's stream: a GPU path tracer reusing the walks (the reference's
// spectral kernel calls traverseClosest / traverseAny, spectral_kernel.js:288,
// 451).
static sb_status device_query_ready(sb_ctx* ctx) {
    if (!ctx->sceneLoaded || ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "scene / TLAS not ready");
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    return flat_if_needed(ctx);
}

sb_status sb_raycast_device(sb_ctx* ctx, const float* ro, const float* rd, uint32_t n, float* tOut, int32_t* triOut,
                            int32_t* instOut) {
    if (!ctx || (n && (!ro || !rd || !tOut || !triOut || !instOut))) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (n == 0) return ctx->sceneLoaded ? SB_OK : fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    sb_status s = device_query_ready(ctx);
    if (s != SB_OK) return s;
    CK(launch_raycast(dev_scene(ctx), ro, rd, n, tOut, triOut, instOut, ctx->dErr, ctx->stream));
    return SB_OK;
}

sb_status sb_occluded_device(sb_ctx* ctx, const float* ro, const float* rd, const float* maxDist, uint32_t n,
                             uint8_t* blockedOut) {
    if (!ctx || (n && (!ro || !rd || !maxDist || !blockedOut))) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (n == 0) return ctx->sceneLoaded ? SB_OK : fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    sb_status s = device_query_ready(ctx);
    if (s != SB_OK) return s;
    CK(launch_occluded(dev_scene(ctx), ro, rd, maxDist, n, blockedOut, ctx->dErr, ctx->stream));
    return SB_OK;
}

sb_status sb_probe_rays(sb_ctx* ctx, uint32_t cascade, uint32_t probeOffset, uint32_t updatedCount, float* roOut,
                        float* rdOut) {
    if (!ctx || (updatedCount && (!roOut || !rdOut))) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (cascade >= SB_MAX_CASCADES || !ctx->casc[cascade].configured)
        return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", cascade);
    const Cascade& K = ctx->casc[cascade];
    if (updatedCount > K.probeTotal || probeOffset >= K.probeTotal)
        return fail(ctx, SB_ERR_INVALID_ARG, "probe range outside the cascade");
    if (updatedCount == 0) return SB_OK;
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)updatedCount * K.grid.raysPerProbe;
    float *dro = nullptr, *drd = nullptr;
    CK(cudaMallocAsync(&dro, n * 12, ctx->stream));
    CK(cudaMallocAsync(&drd, n * 12, ctx->stream));
    CK(launch_probe_rays(dev_cascade(ctx, cascade, probeOffset, updatedCount), ctx->params.frameJitter, dro, drd,
                         ctx->stream));
    CK(cudaMemcpyAsync(roOut, dro, n * 12, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(rdOut, drd, n * 12, cudaMemcpyDeviceToHost, ctx->stream));
    cudaFreeAsync(dro, ctx->stream);
    cudaFreeAsync(drd, ctx->stream);
    return sb_synchronize(ctx);
}

sb_status sb_build_blas_device(sb_ctx* ctx, const float* positions, uint32_t vertexCount, const uint32_t* indices,
                               uint32_t triCount, uint32_t leafSize, uint32_t* nodesOut, uint32_t* triOrderOut,
                               uint32_t* nodeCountOut) {
    if (!ctx || !positions || !indices || !nodesOut || !triOrderOut || !nodeCountOut)
        return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (triCount == 0 || vertexCount == 0) return fail(ctx, SB_ERR_INVALID_ARG, "empty mesh");
    if (leafSize == 0 || leafSize > 255) return fail(ctx, SB_ERR_INVALID_ARG, "leaf size %u: 1..255", leafSize);
    if (triCount >= (1u << 24)) return fail(ctx, SB_ERR_INVALID_ARG, "%u triangles: the leaf offset has 24 bits", triCount);
    cudaSetDevice(ctx->device);
    if (!ctx->builder) ctx->builder = blas_builder_create();
    CK(blas_build(ctx->builder, positions, vertexCount, indices, triCount, leafSize, nodesOut, triOrderOut,
                  nodeCountOut, ctx->dErr, ctx->stream));
    return SB_OK;
}

sb_status sb_build_blas_gpu(sb_ctx* ctx, const float* pos3, uint32_t vertexCount, const uint32_t* index3,
                            uint32_t triCount, uint32_t leafSize, uint32_t* nodesOut, uint32_t* triOrderOut,
                            uint32_t* nodeCountOut) {
    if (!ctx || !pos3 || !index3 || !nodesOut || !triOrderOut || !nodeCountOut)
        return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (triCount == 0 || vertexCount == 0) return fail(ctx, SB_ERR_INVALID_ARG, "empty mesh");
    for (size_t i = 0; i < (size_t)triCount * 3; ++i)
        if (index3[i] >= vertexCount) return fail(ctx, SB_ERR_INVALID_ARG, "triangle %zu: vertex index out of range", i / 3);
    cudaSetDevice(ctx->device);
    float* dp = nullptr;
    uint32_t *di = nullptr, *dn = nullptr, *dord = nullptr, *dc = nullptr;
    CK(cudaMallocAsync(&dp, (size_t)vertexCount * 12, ctx->stream));
    CK(cudaMallocAsync(&di, (size_t)triCount * 12, ctx->stream));
    CK(cudaMallocAsync(&dn, (size_t)triCount * 64, ctx->stream));
    CK(cudaMallocAsync(&dord, (size_t)triCount * 4, ctx->stream));
    CK(cudaMallocAsync(&dc, 4, ctx->stream));
    CK(cudaMemcpyAsync(dp, pos3, (size_t)vertexCount * 12, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(di, index3, (size_t)triCount * 12, cudaMemcpyHostToDevice, ctx->stream));
    sb_status s = sb_build_blas_device(ctx, dp, vertexCount, di, triCount, leafSize, dn, dord, dc);
    uint32_t count = 0;
    if (s == SB_OK) {
        CK(cudaMemcpyAsync(&count, dc, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (count == 0 || count > 2 * triCount) s = fail(ctx, SB_ERR_CUDA, "BLAS build produced %u nodes", count);
    }
    if (s == SB_OK) {
        CK(cudaMemcpyAsync(nodesOut, dn, (size_t)count * 32, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(triOrderOut, dord, (size_t)triCount * 4, cudaMemcpyDeviceToHost, ctx->stream));
        *nodeCountOut = count;
    }
    cudaFreeAsync(dp, ctx->stream); cudaFreeAsync(di, ctx->stream); cudaFreeAsync(dn, ctx->stream);
    cudaFreeAsync(dord, ctx->stream); cudaFreeAsync(dc, ctx->stream);
    if (s != SB_OK) return s;
    return sb_synchronize(ctx);
}

sb_status sb_fit_fine_box(sb_ctx* ctx, const double boxMin[3], const double boxSize[3], double outMin[3],
                          double outSize[3], int32_t* found) {
    if (!ctx || !boxMin || !boxSize || !outMin || !outSize || !found) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    *found = 0;
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    cudaSetDevice(ctx->device);
    if (!ctx->dHist) CK(cudaMalloc(&ctx->dHist, 4096 * sizeof(uint32_t)));
    double inv[3];
    for (int a = 0; a < 3; ++a) inv[a] = 16.0 / std::fmax(1e-6, boxSize[a]);
    CK(launch_fine_hist(ctx->B, boxMin, inv, ctx->dHist, ctx->stream));
    std::vector<uint32_t> h(4096);
    CK(cudaMemcpyAsync(h.data(), ctx->dHist, 4096 * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    sb_status s = sb_synchronize(ctx);
    if (s != SB_OK) return s;
    *found = fine_box_from_hist(h.data(), boxMin, boxSize, outMin, outSize) ? 1 : 0;
    return SB_OK;
}

void sb_gather_params_defaults(sb_gather_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->normalBias[0] = p->normalBias[1] = 0.04f;
    p->detailStrength = 1.0f;
    p->intensity = 1.0f;
    p->enabled = 1.0f;
    p->samplePositionScale = 1.0f;
    p->sampleBiasScale = 1.0f;
    p->borderBand = 0.15f;
    p->cascades = 1;
    p->reflectionIntensity = 1.0f;
    p->roughnessLimit = 1.0f;
}

// Validates a gather's arguments and fills its launch arguments.
static sb_status gather_args(sb_ctx* ctx, const sb_gather_params* prm, const float* position, const float* stableNormal,
                             const float* detailNormal, uint32_t count, float* out, GatherArgs& A) {
    if (!ctx || !prm || (count && (!position || !stableNormal || !detailNormal || !out)))
        return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!aligned(position) || !aligned(stableNormal) || !aligned(detailNormal) || !aligned(out))
        return fail(ctx, SB_ERR_INVALID_ARG, "gather arrays must be 16-byte aligned float4 arrays");
    if (prm->cascades < 1 || prm->cascades > 2) return fail(ctx, SB_ERR_INVALID_ARG, "cascades must be 1 or 2");
    if (prm->cascades == 2 && prm->dualDetail) return fail(ctx, SB_ERR_INVALID_ARG, "dual detail needs one cascade");
    for (uint32_t c = 0; c < prm->cascades; ++c)
        if (!ctx->casc[c].configured || !ctx->casc[c].atlas)
            return fail(ctx, SB_ERR_NOT_READY, "cascade %u not configured", c);
    A = GatherArgs{};
    for (uint32_t c = 0; c < prm->cascades; ++c) {
        const Cascade& K = ctx->casc[c];
        for (int a = 0; a < 3; ++a) {
            A.c[c].gridMin[a] = K.grid.gridMin[a];
            A.c[c].gridSize[a] = K.grid.gridSize[a];
            A.c[c].res[a] = float(K.grid.res[a]);
        }
        A.c[c].atlasW = K.atlasW;
        A.c[c].atlasH = K.atlasH;
        A.c[c].atlas = K.atlas;
        A.c[c].depth = K.depthAtlas;
        A.c[c].rough = K.roughAtlas;
        A.c[c].glossy = K.reflTier >= SB_REFLECT_HIGH ? K.glossyAtlas : nullptr;
        A.c[c].glossyOct = K.glossyOct;
        A.c[c].glossyTile = K.glossyTile;
        A.c[c].glossyTilesX = K.glossyTilesX;
        A.c[c].glossyW = K.glossyTilesX * K.glossyTile;
        A.c[c].glossyH = K.glossyTilesY * K.glossyTile;
    }
    A.cascades = prm->cascades;
    A.dualDetail = prm->dualDetail ? 1u : 0u;
    A.count = count;
    A.normalBias0 = prm->normalBias[0];
    A.chebyBias[0] = prm->chebyBias[0];
    A.chebyBias[1] = prm->chebyBias[1];
    A.chebyStrength = prm->chebyStrength;
    A.detailStrength = prm->detailStrength;
    A.intensity = prm->intensity;
    A.enabled = prm->enabled;
    A.samplePositionScale = prm->samplePositionScale;
    A.sampleBiasScale = prm->sampleBiasScale;
    A.borderBand = prm->borderBand;
    A.reflectionIntensity = prm->reflectionIntensity;
    A.roughnessLimit = prm->roughnessLimit;
    A.position = reinterpret_cast<const float4*>(position);
    A.stableNormal = reinterpret_cast<const float4*>(stableNormal);
    A.detailNormal = reinterpret_cast<const float4*>(detailNormal);
    A.out = reinterpret_cast<float4*>(out);
    return SB_OK;
}

sb_status sb_gather_irradiance(sb_ctx* ctx, const sb_gather_params* prm, const float* position,
                               const float* stableNormal, const float* detailNormal, uint32_t count, float* out) {
    GatherArgs A;
    sb_status s = gather_args(ctx, prm, position, stableNormal, detailNormal, count, out, A);
    if (s != SB_OK || count == 0) return s;
    cudaSetDevice(ctx->device);
    CK(launch_gather(A, ctx->stream));
    return SB_OK;
}

sb_status sb_gather_reflections(sb_ctx* ctx, const sb_gather_params* prm, const float* position,
                                const float* stableNormal, const float* detailNormal, const float* reflection,
                                uint32_t count, float* outIrradiance, float* outReflection) {
    GatherArgs A;
    sb_status s = gather_args(ctx, prm, position, stableNormal, detailNormal, count, outIrradiance, A);
    if (s != SB_OK) return s;
    if (count && (!reflection || !outReflection)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if ((reinterpret_cast<uintptr_t>(reflection) & 15u) || (reinterpret_cast<uintptr_t>(outReflection) & 15u))
        return fail(ctx, SB_ERR_INVALID_ARG, "gather arrays must be 16-byte aligned float4 arrays");
    for (uint32_t c = 0; c < prm->cascades; ++c)
        if (!ctx->casc[c].roughAtlas)
            return fail(ctx, SB_ERR_NOT_READY, "cascade %u has no reflection lobes (sb_set_reflection_quality)", c);
    if (prm->cascades == 2 && (ctx->casc[0].reflTier >= SB_REFLECT_HIGH) != (ctx->casc[1].reflTier >= SB_REFLECT_HIGH))
        return fail(ctx, SB_ERR_NOT_READY, "the cascades' reflection tiers differ");
    if (count == 0) return SB_OK;
    cudaSetDevice(ctx->device);
    A.reflection = reinterpret_cast<const float4*>(reflection);
    A.outReflection = reinterpret_cast<float4*>(outReflection);
    CK(launch_gather_combined(A, ctx->stream));
    return SB_OK;
}

sb_status sb_occluded(sb_ctx* ctx, const float* ro, const float* rd, const float* maxDist, uint32_t n, uint8_t* out) {
    if (!ctx || (n && (!ro || !rd || !maxDist || !out))) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!ctx->sceneLoaded || ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "scene / TLAS not ready");
    if (n == 0) return SB_OK;
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    s = flat_if_needed(ctx);
    if (s != SB_OK) return s;
    float *dro = nullptr, *drd = nullptr, *dm = nullptr;
    uint8_t* dout = nullptr;
    CK(cudaMallocAsync(&dro, (size_t)n * 12, ctx->stream));
    CK(cudaMallocAsync(&drd, (size_t)n * 12, ctx->stream));
    CK(cudaMallocAsync(&dm, (size_t)n * 4, ctx->stream));
    CK(cudaMallocAsync(&dout, (size_t)n, ctx->stream));
    CK(cudaMemcpyAsync(dro, ro, (size_t)n * 12, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(drd, rd, (size_t)n * 12, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dm, maxDist, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_occluded(dev_scene(ctx), dro, drd, dm, n, dout, ctx->dErr, ctx->stream));
    CK(cudaMemcpyAsync(out, dout, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    cudaFreeAsync(dro, ctx->stream); cudaFreeAsync(drd, ctx->stream); cudaFreeAsync(dm, ctx->stream);
    cudaFreeAsync(dout, ctx->stream);
    return sb_synchronize(ctx);
}

// ----------------------------------------------------------- refit / TLAS
sb_status sb_refit_blas(sb_ctx* ctx, uint32_t root, uint32_t end) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ++ctx->epoch;
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    if (!(end > root && end <= ctx->B.nodeCount))
        return fail(ctx, SB_ERR_LAYOUT_VIOLATION, "refit range [%u,%u) outside the node pool", root, end);
    cudaSetDevice(ctx->device);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    // a range checked on the current layout refits with the bottom-up pass alone
    int slot = -1;
    for (int k = 0; k < 16; ++k) {
        const auto& r = ctx->refitRanges[k];
        if (r.used && r.root == root && r.end == end && r.epoch == ctx->packEpoch) slot = k;
    }
    const bool validated = slot >= 0;
    if (!validated) {
        // relinking rewrites the parents of [root, end): overlapping cached ranges are stale
        for (auto& r : ctx->refitRanges)
            if (r.used && r.root < end && root < r.end) r.used = false;
        slot = (int)(ctx->refitNext++ % 16u);
        ctx->refitRanges[slot] = {root, end, ctx->packEpoch, true};
    }
    CK(launch_refit_blas(ctx->B, root, end, ctx->dErr, ctx->dGate + slot, ctx->stream, validated));
    ctx->flat.mark_blas_range(root, end);  // its instances leave the scene BVH
    return SB_OK;
}

// Index of the first of `count` 16-double matrices holding a NaN or an
// infinity, or `count` when all are finite. A non-finite world matrix would
// give NaN instance rows, bounds and TLAS build keys.
static uint32_t first_nonfinite_matrix(const double* world16, uint32_t count) {
    for (uint32_t i = 0; i < count; ++i)
        for (int k = 0; k < 16; ++k)
            if (!std::isfinite(world16[(size_t)i * 16 + k])) return i;
    return count;
}

sb_status sb_set_instances(sb_ctx* ctx, uint32_t count, const double* world16, const uint8_t* active,
                           const uint32_t* blasRoot, const uint32_t* blasEnd) {
    if (!ctx || !world16 || !active || !blasRoot || !blasEnd) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    if (count != ctx->B.instCount)
        return fail(ctx, SB_ERR_INVALID_ARG, "instance count %u != scene instCount %u", count, ctx->B.instCount);
    for (uint32_t i = 0; i < count; ++i)
        if (!(blasRoot[i] < blasEnd[i] && blasEnd[i] <= ctx->B.nodeCount))
            return fail(ctx, SB_ERR_LAYOUT_VIOLATION, "instance %u BLAS range [%u,%u) invalid", i, blasRoot[i], blasEnd[i]);
    if (uint32_t bad = first_nonfinite_matrix(world16, count); bad < count)
        return fail(ctx, SB_ERR_INVALID_ARG, "instance %u world matrix is not finite", bad);
    ++ctx->epoch;
    ++ctx->structGen;
    cudaSetDevice(ctx->device);
    InstanceTable& I = ctx->I;
    if (!ctx->instancesSet || I.count != count) {
        release(I.world); release(I.active); release(I.blasRoot); release(I.blasEnd); release(I.aabb);
        release(I.invRows); release(I.detSign); release(I.order); release(I.slotOf); release(I.liveBounds);
        release(I.nodeDepth); release(I.scratch); release(ctx->instOwner);
        size_t c;
        c = 0; CK(grow(I.world, c, (size_t)count * 16));
        c = 0; CK(grow(I.active, c, (size_t)count));
        c = 0; CK(grow(I.blasRoot, c, (size_t)count));
        c = 0; CK(grow(I.blasEnd, c, (size_t)count));
        c = 0; CK(grow(I.aabb, c, (size_t)count * 9));
        c = 0; CK(grow(I.invRows, c, (size_t)count * 12));
        c = 0; CK(grow(I.detSign, c, (size_t)count));
        c = 0; CK(grow(I.order, c, (size_t)count));
        c = 0; CK(grow(I.slotOf, c, (size_t)count));
        c = 0; CK(grow(I.liveBounds, c, (size_t)count * 6));
        c = 0; CK(grow(I.nodeDepth, c, (size_t)ctx->B.tlasNodeCount));
        c = 0; CK(grow(I.scratch, c, (size_t)4));
        c = 0; CK(grow(ctx->instOwner, c, (size_t)count));
        I.count = count;
    }
    CK(cudaMemcpyAsync(I.world, world16, (size_t)count * 128, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(I.active, active, count, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(I.blasRoot, blasRoot, (size_t)count * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(I.blasEnd, blasEnd, (size_t)count * 4, cudaMemcpyHostToDevice, ctx->stream));
    ctx->instancesSet = true;
    ctx->flat.invalidate();
    if (!ctx->tlasPending) {
        // the uploaded TLAS stays; derive the slot maps from it on the next pack
        ctx->needPack = true;
    }
    return SB_OK;
}

sb_status sb_build_tlas(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ++ctx->epoch;
    ++ctx->structGen;
    if (!ctx->instancesSet) return fail(ctx, SB_ERR_NOT_READY, "sb_set_instances first");
    if (ctx->I.count > TLAS_BUILD_MAX)
        return fail(ctx, SB_ERR_UNSUPPORTED, "%u instances > %u (single-CTA TLAS build)", ctx->I.count, TLAS_BUILD_MAX);
    cudaSetDevice(ctx->device);
    uint32_t nodes = tlas_nodes_for(ctx->I.count);
    if (nodes != ctx->B.tlasNodeCount)
        return fail(ctx, SB_ERR_INVALID_ARG, "TLAS capacity %u != %u nodes", ctx->B.tlasNodeCount, nodes);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    CK(launch_tlas_build(ctx->B, ctx->I, ctx->dErr, ctx->stream));
    CK(launch_tlas_pairs(ctx->B, ctx->stream));
    ctx->flat.invalidate();
    ctx->tlasPending = false;
    ctx->tlasOnDevice = true;
    return SB_OK;
}

sb_status sb_update_transforms(sb_ctx* ctx, const uint32_t* src, const double* world16, uint32_t count) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ++ctx->epoch;
    if (!ctx->instancesSet || ctx->tlasPending) return fail(ctx, SB_ERR_NOT_READY, "instances / TLAS not ready");
    if (!ctx->tlasOnDevice)
        return fail(ctx, SB_ERR_NOT_READY, "the transform lane needs the slot order of a TLAS built by sb_build_tlas");
    if (count && (!src || !world16)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(ctx->device);
    for (uint32_t i = 0; i < count; ++i)
        if (src[i] >= ctx->I.count) return fail(ctx, SB_ERR_INVALID_ARG, "instance %u out of range", src[i]);
    if (uint32_t bad = count ? first_nonfinite_matrix(world16, count) : 0u; bad < count)
        return fail(ctx, SB_ERR_INVALID_ARG, "instance %u world matrix is not finite", src[bad]);
    sb_status s = pack_if_needed(ctx);
    if (s != SB_OK) return s;
    if (count) {
        if (count > ctx->stageCap) {
            release(ctx->dStage); release(ctx->dStageM);
            size_t c = 0;
            CK(grow(ctx->dStage, c, (size_t)count));
            c = 0;
            CK(grow(ctx->dStageM, c, (size_t)count * 16));
            ctx->stageCap = count;
        }
        CK(cudaMemcpyAsync(ctx->dStage, src, (size_t)count * 4, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->dStageM, world16, (size_t)count * 128, cudaMemcpyHostToDevice, ctx->stream));
        CK(launch_update_refit_tlas(ctx->B, ctx->I, ctx->dStage, ctx->dStageM, count, 1, ctx->dErr, ctx->stream));
        for (uint32_t i = 0; i < count; ++i) ctx->flat.mark_source(src[i]);  // moved: out of the scene BVH
    } else {
        // rewriteInstanceRows:false — bounds from the (refit) BLAS roots
        CK(launch_update_refit_tlas(ctx->B, ctx->I, nullptr, nullptr, 0, 0, ctx->dErr, ctx->stream));
    }
    return SB_OK;
}

// ---------------------------------------------------------------- stats
sb_status sb_enable_counters(sb_ctx* ctx, int32_t on) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ctx->countersOn = on != 0;
    return SB_OK;
}

sb_status sb_rebuild_scene_bvh(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    ctx->flat.invalidate();
    return SB_OK;
}

sb_status sb_set_scene_bvh_build_mode(sb_ctx* ctx, uint32_t mode) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    if (mode > SB_SCENE_BVH_BACKGROUND) return fail(ctx, SB_ERR_INVALID_ARG, "scene BVH build mode %u", mode);
    ctx->flat.background = mode == SB_SCENE_BVH_BACKGROUND;
    return SB_OK;
}

sb_status sb_finish_scene_bvh(sb_ctx* ctx) {
    if (!ctx) return SB_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::string why;
    CK(ctx->flat.finish(ctx->stream, why));
    return SB_OK;
}

sb_status sb_get_stats(sb_ctx* ctx, sb_stats* out) {
    if (!ctx || !out) return SB_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof *out);
    out->sceneBvhBuilds = ctx->flat.builds;
    out->sceneBvhActive = ctx->flat.enabled && ctx->flat.ready && !ctx->flat.overflowed ? 1u : 0u;
    out->sceneBvhBuilding = ctx->flat.building() ? 1u : 0u;
    out->lastSceneBvhBuildMs = ctx->flat.lastBuildMs;
    cudaSetDevice(ctx->device);
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->countersOn) {
        unsigned long long c[16];
        CK(cudaMemcpy(c, ctx->dCounters, sizeof c, cudaMemcpyDeviceToHost));
        out->primaryRays = c[0];
        out->shadowRays = c[1];
        out->tlasNodeVisits = c[2] + c[6];
        out->instanceVisits = c[3] + c[7];
        out->blasNodeVisits = c[4] + c[8];
        out->triangleTests = c[5] + c[9];
        out->shadowTlasNodeVisits = c[6];
        out->shadowInstanceVisits = c[7];
        out->shadowBlasNodeVisits = c[8];
        out->shadowTriangleTests = c[9];
    }
    if (ctx->timed && ctx->lastWasGraph) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) out->lastSolveMs = ms;  // whole frame
    } else if (ctx->timed) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) out->lastSolveMs = ms;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->evMid) == cudaSuccess) out->lastTraceMs = ms;
        if (cudaEventElapsedTime(&ms, ctx->evMid, ctx->ev1) == cudaSuccess) out->lastBlendMs = ms;
        if (ctx->singleChunk) {
            if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->evC) == cudaSuccess) out->lastPrimaryMs = ms;
            if (cudaEventElapsedTime(&ms, ctx->evC, ctx->evA) == cudaSuccess) out->lastEmitMs = ms;
            if (cudaEventElapsedTime(&ms, ctx->evA, ctx->evB) == cudaSuccess) out->lastShadowMs = ms;
            if (cudaEventElapsedTime(&ms, ctx->evB, ctx->evMid) == cudaSuccess) out->lastShadeMs = ms;
        }
    }
    float fms = 0.0f;
    if (ctx->tape.timedF && cudaEventElapsedTime(&fms, ctx->tape.evF0, ctx->tape.evF1) == cudaSuccess)
        out->lastForwardRecordMs = fms;
    if (ctx->tape.timedB && cudaEventElapsedTime(&fms, ctx->tape.evB0, ctx->tape.evB1) == cudaSuccess)
        out->lastBackwardMs = fms;
    out->kernelLaunches = launches();
    return SB_OK;
}

sb_status sb_get_tuning(const sb_ctx* ctx, sb_tuning* out) {
    if (!ctx || !out) return SB_ERR_INVALID_ARG;
    out->traceBlock = ctx->tune.block;
    out->sortKey = ctx->tune.sortKey;
    out->smemTlasNodes = ctx->tune.smemTlasNodes;
    out->bvhKind = ctx->bvhKind;
    out->smemWideNodes = ctx->tune.smemWideNodes;
    return SB_OK;
}

sb_status sb_set_tuning(sb_ctx* ctx, const sb_tuning* t) {
    if (!ctx || !t) return SB_ERR_INVALID_ARG;
    if (t->traceBlock == 0 || t->traceBlock > 256 || t->traceBlock % 32)
        return fail(ctx, SB_ERR_INVALID_ARG, "traceBlock %u: multiple of 32 in [32,256]", t->traceBlock);
    if (t->bvhKind > 2) return fail(ctx, SB_ERR_UNSUPPORTED, "bvhKind %u not built", t->bvhKind);
    if (t->smemWideNodes > 512)
        return fail(ctx, SB_ERR_INVALID_ARG, "smemWideNodes %u > 512 (80 bytes each)", t->smemWideNodes);
    if (t->sortKey > 3) return fail(ctx, SB_ERR_INVALID_ARG, "sortKey %u: 0, 1, 2 or 3", t->sortKey);
    if (t->bvhKind != ctx->bvhKind) ctx->flat.invalidate();
    ctx->tune.smemWideNodes = t->smemWideNodes;
    ctx->bvhKind = t->bvhKind;
    ++ctx->structGen;
    ctx->tune.block = t->traceBlock;
    ctx->tune.sortKey = t->sortKey;
    ctx->tune.smemTlasNodes = t->smemTlasNodes;
    return SB_OK;
}

}  // extern "C"

extern "C" sb_status sb_update_deform(sb_ctx* ctx, uint32_t vertexStart, uint32_t vertexCount,
                                      const float* vertexData, uint32_t root, uint32_t end) {
    if (!ctx || (vertexCount && !vertexData)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    ++ctx->epoch;
    if ((uint64_t)vertexStart + vertexCount > ctx->B.vertexCount)
        return fail(ctx, SB_ERR_INVALID_ARG, "vertex range [%u,+%u) outside the pool", vertexStart, vertexCount);
    cudaSetDevice(ctx->device);
    CK(cudaMemcpyAsync(ctx->B.vertexData + (size_t)vertexStart * 8, vertexData, (size_t)vertexCount * 32,
                       cudaMemcpyHostToDevice, ctx->stream));
    return sb_refit_blas(ctx, root, end);
}

extern "C" sb_status sb_update_deform_xyz(sb_ctx* ctx, uint32_t vertexStart, uint32_t vertexCount,
                                          const float* positions, const float* normals, uint32_t root,
                                          uint32_t end) {
    if (!ctx || (vertexCount && !positions)) return fail(ctx, SB_ERR_INVALID_ARG, "null argument");
    if (!ctx->sceneLoaded) return fail(ctx, SB_ERR_NOT_READY, "no scene uploaded");
    if ((uint64_t)vertexStart + vertexCount > ctx->B.vertexCount)
        return fail(ctx, SB_ERR_INVALID_ARG, "vertex range [%u,+%u) outside the pool", vertexStart, vertexCount);
    ++ctx->epoch;
    cudaSetDevice(ctx->device);
    const size_t n = vertexCount, floats = n * (normals ? 6u : 3u);
    // the previous call's copy must have read the page-locked buffer before it is refilled
    if (ctx->deformPending) CK(cudaEventSynchronize(ctx->evDeform));
    ctx->deformPending = false;
    if (floats > ctx->deformCap) {
        if (ctx->hDeform) cudaFreeHost(ctx->hDeform);
        if (ctx->dDeform) cudaFree(ctx->dDeform);
        ctx->hDeform = nullptr;
        ctx->dDeform = nullptr;
        ctx->deformCap = 0;
        CK(cudaHostAlloc((void**)&ctx->hDeform, floats * sizeof(float), cudaHostAllocDefault));
        CK(cudaMalloc((void**)&ctx->dDeform, floats * sizeof(float)));
        ctx->deformCap = floats;
    }
    if (!ctx->evDeform) CK(cudaEventCreateWithFlags(&ctx->evDeform, cudaEventDisableTiming));
    if (n) {
        std::memcpy(ctx->hDeform, positions, n * 3 * sizeof(float));
        if (normals) std::memcpy(ctx->hDeform + 3 * n, normals, n * 3 * sizeof(float));
        CK(cudaMemcpyAsync(ctx->dDeform, ctx->hDeform, floats * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaEventRecord(ctx->evDeform, ctx->stream));
        ctx->deformPending = true;
        CK(launch_scatter_vertices(ctx->B.vertexData + (size_t)vertexStart * 8, ctx->dDeform,
                                   normals ? ctx->dDeform + 3 * n : nullptr, vertexCount, ctx->stream));
    }
    return sb_refit_blas(ctx, root, end);
}
