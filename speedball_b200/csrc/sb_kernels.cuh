// sb_kernels.cuh — launcher declarations shared by the host side (sb_ctx.cu).
#pragma once
#include "sb_internal.cuh"

namespace sb {

// Process-wide count of kernels this library launched (reported in sb_stats).
void note_launch();
uint64_t launches();

// The closest-hit stage on the 8-wide tree hands each lane a new ray as soon
// as its walk ends (per-lane refill) instead of running fixed 32-ray batches
// per warp; 0 keeps the batches (and with them the costliest-first order).
#ifndef SB_PRIMARY_REFILL
#define SB_PRIMARY_REFILL 1
#endif

struct TraceTuning {
    uint32_t block;          // threads per block of the trace kernel
    uint32_t smemTlasNodes;  // stage the TLAS in shared memory when it has at most this many nodes
    uint32_t sortKey;        // ray issue order: 0 direction-major, 1 probe-major, 2 direction-major over probe
                             // tiles, 3 as 2 with closest-hit batches costliest first (last full solve's cycles)
    int numSms;
    uint32_t smemWideNodes;  // top 8-wide scene-BVH nodes staged in shared memory per closest-hit CTA
};

// Scene buffers in the reference layouts plus the derived layouts.
struct SceneBuffers {
    uint32_t* nodes = nullptr;        // nodeCount*8
    uint32_t* triIndex = nullptr;     // triCount*3
    float* vertexData = nullptr;      // vertexCount*8
    uint32_t* triMaterial = nullptr;  // triCount
    float* materials = nullptr;       // materialsLen
    float* lights = nullptr;          // lightsLen
    float4* lightGates = nullptr;     // derived, 64 x 3 (light_gates)
    float4* tris = nullptr;           // derived, triCount*3
    float4* inst = nullptr;           // derived, instCount*4
    uint4* tlas = nullptr;            // derived, tlasNodeCount*2
    uint32_t* matBits = nullptr;      // derived, per material accept bits
    uint4* pairs = nullptr;           // derived, nodeCount*4: child-pair nodes of the BLASes
    uint4* tlasPairs = nullptr;       // derived, tlasNodeCount*4: child-pair nodes of the TLAS
    uint32_t* depth = nullptr;        // 2 words: deepest BLAS / TLAS node (DEPTH_UNKNOWN = no pairs)
    uint32_t* parent = nullptr;       // nodeCount: parent of each BLAS node (refit)
    uint32_t* arrive = nullptr;       // nodeCount: refit arrival counters
    uint32_t* subRoots = nullptr;     // nodeCount: roots of the refit's CTA subtrees, per range from its root
    uint32_t* valid = nullptr;        // 1 word
    uint32_t nodeCount = 0, triCount = 0, vertexCount = 0, materialsLen = 0, materialCount = 0;
    uint32_t instBase = 0, instCount = 0, tlasBase = 0, tlasNodeCount = 0, lightsLen = 0;
};

// The three trace stages over probe slots [slotBegin, slotBegin + slotCount);
// `jobs` holds up to jobCap shadow-ray jobs (32 bytes each).
cudaError_t launch_trace(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t* err,
                         unsigned long long* counters, uint32_t* work, const TraceTuning& tune, cudaStream_t st,
                         float4* jobs, uint32_t jobCap, uint32_t slotBegin, uint32_t slotCount,
                         cudaEvent_t afterPrimary = nullptr, cudaEvent_t afterShadow = nullptr,
                         cudaEvent_t afterClosest = nullptr);
cudaError_t launch_blend_upload(const DevCascade& C, const DevParams& P, cudaStream_t st);
// Positions (and normals when given), 3 floats per vertex, into the first six
// floats of n pooled 8-float vertices.
cudaError_t launch_scatter_vertices(float* vertexData8, const float* positions, const float* normals, uint32_t n,
                                    cudaStream_t st);
cudaError_t launch_glossy(const DevCascade& C, const DevParams& P, cudaStream_t st);
cudaError_t launch_shade(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t slotCount,
                         cudaStream_t st);

// Batched stages (every item of B in one launch per stage). B.work must hold
// 3 words; every item's W.jobs / W.jobCap / W.work are the batch's shared ones.
cudaError_t launch_trace_batch(const BatchArgs& B, const TraceTuning& tune, cudaStream_t st,
                               cudaEvent_t afterPrimary = nullptr, cudaEvent_t afterShadow = nullptr,
                         cudaEvent_t afterClosest = nullptr);
cudaError_t launch_blend_upload_batch(const BatchArgs& B, cudaStream_t st);
uint32_t blend_blocks(uint32_t updatedCount);  // CTAs of the blend for one solve
// The batched kernels (stage 0 primary, 1 emit, 2 shadow, 3 shade; blend):
// a captured graph refreshes their BatchArgs parameter on every replay.
const void* trace_batch_kernel(int stage);
const void* blend_batch_kernel();

// Adjoint of shade + blend + upload (sb_adjoint.cu), over every probe of a
// cascade (probe slot = probe index). Gradient layouts: gE / E per interior
// texel (36 per probe, probe-major), gH per history texel (64 per probe: rgb,
// m2), gA per atlas texel (rgb), gR per ray (rgb), gParam in doubles:
// [albedo materialCount*3 | emissive materialCount*3 | light scale lightCount].
cudaError_t launch_adjoint_loss(const float4* E, const float* target, uint32_t n, float4* gE, double* loss,
                                cudaStream_t st);
cudaError_t launch_upload_bwd(const DevCascade& C, const DevParams& P, const float4* H, const float4* gE,
                              const float4* gA, float4* gH, cudaStream_t st);
cudaError_t launch_blend_bwd(const DevCascade& C, const DevParams& P, const float4* rays, const float4* Hprev,
                             const float4* gH, float4* gHprev, float4* gR, cudaStream_t st);
cudaError_t launch_shade_bwd(const DevScene& S, const DevCascade& C, const DevParams& P, const float4* gR,
                             double* gParam, float4* gA, cudaStream_t st);
cudaError_t launch_light_grid(float* lights, uint32_t lightCount, const DevCascade& g0, cudaStream_t st);
// The 64 light records' gate fields as three aligned float4 each: (position, range),
// (direction, type), (colour, emitter class).
cudaError_t launch_light_gates(const float* lights, float4* gates, cudaStream_t st);
cudaError_t launch_clear_cascade(const DevCascade& C, cudaStream_t st);

// Validation + derived-layout packing (sb_pack.cu).
cudaError_t launch_pack_scene(const SceneBuffers& B, uint32_t* err, cudaStream_t st);
cudaError_t launch_pack_tris(const SceneBuffers& B, uint32_t triBegin, uint32_t triEnd, uint32_t* err, cudaStream_t st);
cudaError_t launch_pack_dynamic(const SceneBuffers& B, uint32_t* err, cudaStream_t st);

// Refit and TLAS lanes (sb_refit.cu). `validated`: the range's parent links
// and layout checks from an earlier call on the same layout are still current
// (their verdict is in *gate, the range's subtree count in gate[16]), so only
// the bottom-up pass runs.
cudaError_t launch_refit_blas(const SceneBuffers& B, uint32_t root, uint32_t end, uint32_t* err, uint32_t* gate,
                              cudaStream_t st, bool validated = false);

struct InstanceTable {
    double* world = nullptr;       // 16 per source instance (column-major)
    uint8_t* active = nullptr;
    uint32_t* blasRoot = nullptr;
    uint32_t* blasEnd = nullptr;
    double* aabb = nullptr;        // 9 per source instance: min, max, centroid
    float* invRows = nullptr;      // 12 per source instance
    float* detSign = nullptr;
    uint32_t* order = nullptr;     // slot -> source
    uint32_t* slotOf = nullptr;    // source -> slot
    float* liveBounds = nullptr;   // 6 per slot
    uint32_t* nodeDepth = nullptr; // TLAS node depth (level-order refit)
    uint32_t* scratch = nullptr;   // TLAS build scratch
    uint32_t count = 0;
    uint32_t maxDepth = 0;
};
constexpr uint32_t TLAS_BUILD_MAX = 4096;  // instances per single-CTA TLAS build

cudaError_t launch_tlas_build(const SceneBuffers& B, const InstanceTable& I, uint32_t* err, cudaStream_t st);
// srcList/world16 are device arrays (count entries); srcList == null updates every
// source instance from its stored matrix (rewriteRows = 0 after a BLAS refit).
cudaError_t launch_update_instances(const SceneBuffers& B, const InstanceTable& I, const uint32_t* srcList,
                                    const double* world16, uint32_t count, int rewriteRows, uint32_t* err,
                                    cudaStream_t st);
cudaError_t launch_tlas_refit(const SceneBuffers& B, const InstanceTable& I, uint32_t* err, cudaStream_t st);
// launch_update_instances followed by launch_tlas_refit, as one single-CTA launch.
cudaError_t launch_update_refit_tlas(const SceneBuffers& B, const InstanceTable& I, const uint32_t* srcList,
                                     const double* world16, uint32_t count, int rewriteRows, uint32_t* err,
                                     cudaStream_t st);
cudaError_t launch_tlas_index(const SceneBuffers& B, const InstanceTable& I, uint32_t* owner, uint32_t* err,
                              cudaStream_t st);

// Child-pair layouts (sb_pairs.cu). launch_blas_pairs derives every BLAS pair
// node and the deepest BLAS node from the reference nodes (structural changes);
// refits keep them current. launch_tlas_pairs does the same for the TLAS after
// a structural TLAS change (pack or build); TLAS refits rewrite their pairs.
cudaError_t launch_blas_pairs(const SceneBuffers& B, cudaStream_t st);
cudaError_t launch_tlas_pairs(const SceneBuffers& B, cudaStream_t st);

// Receiver gather (sb_gather.cu): one cascade's atlases and grid as the gather
// reads them, and one launch's G-buffer.
struct GatherCascade {
    float gridMin[3], gridSize[3], res[3];
    uint32_t atlasW, atlasH;
    const uint2* atlas;   // RGBA16F irradiance atlas
    const uint2* depth;   // RGBA16F depth-moment atlas
    // reflection lobes (combined receiver): rough atlas in the irradiance
    // layout; glossy atlas (null below tier high) of glossyTile-texel tiles
    const uint2* rough;
    const uint2* glossy;
    uint32_t glossyOct, glossyTile, glossyTilesX, glossyW, glossyH;
};
struct GatherArgs {
    GatherCascade c[2];
    uint32_t cascades, dualDetail, count;
    float normalBias0, chebyBias[2], chebyStrength, detailStrength, intensity, enabled;
    float samplePositionScale, sampleBiasScale, borderBand;
    float reflectionIntensity, roughnessLimit;
    const float4* position;
    const float4* stableNormal;
    const float4* detailNormal;
    const float4* reflection;  // combined receiver: direction xyz, roughness w
    float4* out;
    float4* outReflection;
};
cudaError_t launch_gather(const GatherArgs& A, cudaStream_t st);
cudaError_t launch_gather_combined(const GatherArgs& A, cudaStream_t st);
// GPU BLAS build in the threaded layout (sb_build.cu); device scratch lives in
// the builder and grows to the largest mesh built. Out-of-range vertex indices
// latch ERR_LAYOUT.
struct BlasBuilder;
BlasBuilder* blas_builder_create();
void blas_builder_destroy(BlasBuilder* b);
cudaError_t blas_build(BlasBuilder* b, const float* pos, uint32_t V, const uint32_t* idx, uint32_t T,
                       uint32_t leafSize, uint32_t* nodes, uint32_t* order, uint32_t* nodeCount, uint32_t* err,
                       cudaStream_t st);
// Fine-cascade placement (sb_cascade.cu): the 16^3 centroid histogram on the
// GPU, then the box on the host.
cudaError_t launch_fine_hist(const SceneBuffers& B, const double mn[3], const double inv[3], uint32_t* hist,
                             cudaStream_t st);
bool fine_box_from_hist(const uint32_t* hist, const double mn[3], const double size[3], double outMin[3],
                        double outSize[3]);
// emitterVisKernel (sb_trace.cu): one thread per (updated probe, emitter).
cudaError_t launch_emitter_vis(const DevScene& S, const DevCascade& C, const DevParams& P, uint32_t* err,
                               cudaStream_t st);
// The FP32 probe rays of a solve as the trace forms them (sb_probe_rays).
cudaError_t launch_probe_rays(const DevCascade& C, float jitter, float* ro, float* rd, cudaStream_t st);

// Arbitrary-ray queries through the same traversal (raycastFirst-like).
cudaError_t launch_raycast(const DevScene& S, const float* ro, const float* rd, uint32_t n, float* tOut,
                           int32_t* triOut, int32_t* instOut, uint32_t* err, cudaStream_t st);
cudaError_t launch_occluded(const DevScene& S, const float* ro, const float* rd, const float* maxDist, uint32_t n,
                            uint8_t* out, uint32_t* err, cudaStream_t st);

}  // namespace sb
