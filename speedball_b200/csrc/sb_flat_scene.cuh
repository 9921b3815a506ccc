// sb_flat_scene.cuh — a context's scene BVH (layout in sb_flat.h): when it is
// rebuilt, which instance slots it no longer covers, and what the kernels see.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "sb_flat.h"
#include "sb_kernels.cuh"

namespace sb {

struct FlatScene {
    // More moved slots than this: the scene BVH stands aside (`overflowed`) and
    // the traversal walks the reference's TLAS + BLASes, which the GPU refits
    // every frame, until the next rebuild (a structural change, or
    // sb_rebuild_scene_bvh at a moment the host chooses).
    static constexpr uint32_t kMaxDynamic = 256;

    bool enabled = true;  // bvhKind 1 or 2
    bool wide = true;     // bvhKind 1: also the 8-wide tree, which answers closest hits
    bool dirty = true;    // rebuild before the next trace (set through invalidate())
    // Background builds (sb_set_scene_bvh_build_mode): a rebuild reads its
    // inputs back at the next trace, builds on a host thread, and the tree is
    // installed by the first trace after it finished; until then the
    // reference's two-level walk answers. Slots that move meanwhile are marked
    // against the new tree when it is installed.
    bool background = false;
    uint64_t generation = 0;  // structural changes so far: a build of an older one is dropped
    bool ready = false;   // device copy current
    bool overflowed = false;  // more than kMaxDynamic moved slots since the build
    uint64_t builds = 0;      // scene-BVH builds of this context
    uint4* nodes = nullptr;   // binary child-pair tree (any hit; closest hit without `wide`)
    size_t nodeCap = 0;
    uint2* items = nullptr;
    size_t itemCap = 0;
    uint4* wnodes = nullptr;  // 8-wide tree with 8-bit boxes (closest hit)
    size_t wnodeCap = 0;
    uint2* witems = nullptr;
    size_t witemCap = 0;
    bool wideReady = false;
    uint8_t* dSkip = nullptr;
    size_t skipCap = 0;
    uint32_t* dDyn = nullptr;
    size_t dynCap = 0;
    uint32_t root = flat::ENTRY_NONE, depth = 0, itemCount = 0, wideCount = 0, wideDepth = 0;
    std::vector<uint8_t> skip;        // per slot
    std::vector<uint32_t> dyn;        // slots walked through their BLAS
    std::vector<uint32_t> slotRoot, slotEnd, srcToSlot;
    bool marksDirty = false;
    float lastBuildMs = 0.0f;

    // Rebuilds when dirty and uploads pending slot marks. `order` (slot ->
    // source instance, device, may be null) maps transform updates to slots.
    cudaError_t prepare(const SceneBuffers& B, const uint32_t* order, uint32_t orderCount, cudaStream_t st,
                        std::string& why);
    // a structural change: the tree no longer describes the scene
    void invalidate() {
        dirty = true;
        ++generation;
    }
    // true while a background build runs
    bool building() const { return job != nullptr; }
    // wait for a running background build and install it (or drop it when stale)
    cudaError_t finish(cudaStream_t st, std::string& why);
    void mark_source(uint32_t src);
    void mark_blas_range(uint32_t root, uint32_t end);
    void fill(DevScene& S) const;
    void release();

    struct Job;  // one build's inputs and outputs (sb_flat.cu)
    FlatScene();
    ~FlatScene();
    FlatScene(const FlatScene&) = delete;
    FlatScene& operator=(const FlatScene&) = delete;

   private:
    std::unique_ptr<Job> job;  // the running background build, if any
    void mark_slot(uint32_t s);
    cudaError_t snapshot(const SceneBuffers& B, const uint32_t* order, uint32_t orderCount, cudaStream_t st,
                         Job& j);
    cudaError_t install(Job& j, cudaStream_t st, std::string& why);
};

}  // namespace sb
