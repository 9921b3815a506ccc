// sb_flat.cu — building and maintaining a context's scene BVH (sb_flat.h).
//
// A structural change (scene upload, ranged upload of scene buffers, instance
// set, TLAS build) marks the tree dirty; the next trace reads the instance
// records, BLAS nodes, triangle indices and vertices back, forms one item per
// (triangle, active instance slot) with its world-space bounds (the vertices
// under the inverse of the instance's inverse rows, in FP64, widened), builds
// the binned-SAH tree on the host and uploads it. In background mode the build
// runs on a host thread while the traces use the two-level walk, and the first
// trace after it finished installs the tree.
//
// Per frame nothing is rebuilt: a slot whose transform changes, or whose BLAS
// is refit, is marked; the traversal skips that slot's items and walks its
// current BLAS instead. Beyond kMaxDynamic marked slots the tree stands aside
// and the reference's two-level walk (GPU-refit TLAS + BLASes) answers instead.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

#include "sb_flat_scene.cuh"

namespace sb {

namespace {

template <class T>
cudaError_t grow_dev(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

uint32_t f_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Inverse of the affine map local = A * world + b given as three rows (A | b).
bool invert_rows(const float* r, double M[12]) {
    double a[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[3 * i + j] = r[4 * i + j];
    double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
    double inv[9] = {c00 / det, (a[2] * a[7] - a[1] * a[8]) / det, (a[1] * a[5] - a[2] * a[4]) / det,
                     c01 / det, (a[0] * a[8] - a[2] * a[6]) / det, (a[2] * a[3] - a[0] * a[5]) / det,
                     c02 / det, (a[1] * a[6] - a[0] * a[7]) / det, (a[0] * a[4] - a[1] * a[3]) / det};
    const double b[3] = {r[3], r[7], r[11]};
    for (int i = 0; i < 3; ++i) {
        M[4 * i] = inv[3 * i];
        M[4 * i + 1] = inv[3 * i + 1];
        M[4 * i + 2] = inv[3 * i + 2];
        M[4 * i + 3] = -(inv[3 * i] * b[0] + inv[3 * i + 1] * b[1] + inv[3 * i + 2] * b[2]);
    }
    return true;
}

}  // namespace

struct FlatScene::Job {
    // inputs, read back from the device at the start of the build
    uint32_t slots = 0, nodeCount = 0, triCount = 0, vertexCount = 0;
    std::vector<float> inst, vert;
    std::vector<uint32_t> hn, tri;
    std::vector<uint32_t> slotRoot, slotEnd, srcToSlot;
    bool wide = true;
    uint64_t generation = 0;
    std::chrono::steady_clock::time_point t0;
    // slots moved or refit while a background build runs (marked on install)
    std::vector<uint8_t> moved;
    std::vector<uint32_t> movedList;
    bool movedOverflow = false;
    // outputs
    flat::Tree tree;
    flat::WideTree wt;
    bool treeOk = false, wideOk = false;
    uint32_t n = 0;
    std::string why;
    std::thread th;
    std::atomic<bool> done{false};
};

FlatScene::FlatScene() = default;

FlatScene::~FlatScene() {
    if (job && job->th.joinable()) job->th.join();
}

// Reads the instance records, BLAS nodes, triangle indices, vertices and the
// slot order back (synchronizing the stream) and forms the slot tables.
cudaError_t FlatScene::snapshot(const SceneBuffers& B, const uint32_t* order, uint32_t orderCount, cudaStream_t st,
                                Job& j) {
    j.t0 = std::chrono::steady_clock::now();
    j.generation = generation;
    j.wide = wide;
    j.slots = B.instCount;
    j.nodeCount = B.nodeCount;
    j.triCount = B.triCount;
    j.vertexCount = B.vertexCount;
    j.inst.resize((size_t)j.slots * 16);
    j.hn.resize((size_t)B.nodeCount * 8);
    j.tri.resize((size_t)B.triCount * 3);
    j.vert.resize((size_t)B.vertexCount * 8);
    std::vector<uint32_t> ord(orderCount);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && j.slots) e = cudaMemcpy(j.inst.data(), B.inst, j.inst.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && B.nodeCount) e = cudaMemcpy(j.hn.data(), B.nodes, j.hn.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && B.triCount)
        e = cudaMemcpy(j.tri.data(), B.triIndex, j.tri.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && B.vertexCount)
        e = cudaMemcpy(j.vert.data(), B.vertexData, j.vert.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && order && orderCount)
        e = cudaMemcpy(ord.data(), order, ord.size() * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    const uint32_t slots = j.slots;
    j.slotRoot.assign(slots, 0);
    j.slotEnd.assign(slots, 0);
    j.srcToSlot.assign(slots, 0xFFFFFFFFu);
    for (uint32_t s = 0; s < slots; ++s) {
        const uint32_t src = (order && s < orderCount) ? ord[s] : s;
        if (src < slots) j.srcToSlot[src] = s;
        const float* R = j.inst.data() + (size_t)s * 16;
        j.slotRoot[s] = f_bits(R[12]);
        j.slotEnd[s] = f_bits(R[13]);
    }
    j.moved.assign(slots, 0);
    return cudaSuccess;
}

namespace {

// One item per (triangle, active instance slot) with its world-space bounds
// (the vertices under the inverse of the instance's inverse rows, in FP64,
// widened), then the binned-SAH binary tree and the 8-wide tree beside it.
// Host work only: runs on the calling thread or a background one.
void compute(FlatScene::Job& j) {
    const uint32_t slots = j.slots;
    std::vector<uint64_t> slotItems(slots + 1, 0);
    for (uint32_t s = 0; s < slots; ++s) {
        const float* R = j.inst.data() + (size_t)s * 16;
        const uint32_t root = j.slotRoot[s], end = j.slotEnd[s];
        uint64_t c = 0;
        if (R[15] > 0.5f && root < end && end <= j.nodeCount)
            for (uint32_t nd = root; nd < end; ++nd) {
                const uint32_t payload = j.hn[8 * (size_t)nd + 7];
                if (payload != 0xFFFFFFFFu) c += payload >> 24;
            }
        slotItems[s + 1] = slotItems[s] + c;
    }
    const uint64_t cap = slotItems[slots];
    if (cap >= (1ull << 24)) {
        j.why = "scene BVH: too many (triangle, instance) items";
        return;
    }
    std::vector<float> boxes(cap * 6);
    std::vector<uint32_t> itTri(cap), itSlot(cap);
    std::vector<uint8_t> keep(cap, 0);
    std::atomic<uint32_t> nextSlot{0};
    auto work = [&] {
        for (uint32_t s; (s = nextSlot.fetch_add(1)) < slots;) {
            const float* R = j.inst.data() + (size_t)s * 16;
            const uint32_t root = j.slotRoot[s], end = j.slotEnd[s];
            if (slotItems[s + 1] == slotItems[s]) continue;  // inactive or no BLAS
            double M[12];
            if (!invert_rows(R, M)) continue;  // singular: the local test never hits
            uint64_t o = slotItems[s];
            for (uint32_t nd = root; nd < end; ++nd) {
                const uint32_t payload = j.hn[8 * (size_t)nd + 7];
                if (payload == 0xFFFFFFFFu) continue;
                const uint32_t off = payload & 0x00FFFFFFu, cnt = payload >> 24;
                for (uint32_t t = off; t < off + cnt; ++t, ++o) {
                    if (t >= j.triCount) continue;
                    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                    bool ok = true;
                    for (int k = 0; k < 3; ++k) {
                        const uint32_t v = j.tri[3 * (size_t)t + k];
                        if (v >= j.vertexCount) {
                            ok = false;
                            break;
                        }
                        const float* p = j.vert.data() + 8 * (size_t)v;
                        for (int a = 0; a < 3; ++a) {
                            const double w = M[4 * a] * p[0] + M[4 * a + 1] * p[1] + M[4 * a + 2] * p[2] + M[4 * a + 3];
                            lo[a] = std::fmin(lo[a], w);
                            hi[a] = std::fmax(hi[a], w);
                        }
                    }
                    if (!ok || !std::isfinite(lo[0] + lo[1] + lo[2] + hi[0] + hi[1] + hi[2])) continue;
                    // margin well above the FP32 rounding of the local ray and vertices
                    double mag = 0.0, ext = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        mag = std::fmax(mag, std::fmax(std::fabs(lo[a]), std::fabs(hi[a])));
                        ext = std::fmax(ext, hi[a] - lo[a]);
                    }
                    const double m = 1e-5 * mag + 1e-5 * ext + 1e-7;
                    float* bx = boxes.data() + 6 * o;
                    for (int a = 0; a < 3; ++a) bx[a] = std::nextafterf((float)(lo[a] - m), -INFINITY);
                    for (int a = 0; a < 3; ++a) bx[3 + a] = std::nextafterf((float)(hi[a] + m), INFINITY);
                    itTri[o] = t;
                    itSlot[o] = s;
                    keep[o] = 1;
                }
            }
        }
    };
    {
        const unsigned th = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> ts;
        for (unsigned w = 1; w < th && cap > 65536; ++w) ts.emplace_back(work);
        work();
        for (auto& t : ts) t.join();
    }
    // drop degenerate items, keeping slot order
    uint64_t kept = 0;
    for (uint64_t i = 0; i < cap; ++i) {
        if (!keep[i]) continue;
        if (kept != i) {
            std::memcpy(boxes.data() + 6 * kept, boxes.data() + 6 * i, 24);
            itTri[kept] = itTri[i];
            itSlot[kept] = itSlot[i];
        }
        ++kept;
    }
    itTri.resize(kept);
    itSlot.resize(kept);
    const uint32_t n = (uint32_t)itTri.size();
    j.n = n;
    // the 8-wide tree builds beside the binary one
    std::thread wideBuild;
    if (j.wide && n)
        wideBuild = std::thread([&] { j.wideOk = flat::build_wide(boxes.data(), itTri.data(), itSlot.data(), n, j.wt); });
    j.treeOk = flat::build(boxes.data(), itTri.data(), itSlot.data(), n, j.tree);
    if (wideBuild.joinable()) wideBuild.join();
    if (!j.treeOk) j.why = "scene BVH: too many items";
}

}  // namespace

// Uploads a finished build and makes it the tree the walks use.
cudaError_t FlatScene::install(Job& j, cudaStream_t st, std::string& why) {
    (void)st;
    if (!j.treeOk) {
        why = j.why;
        return cudaSuccess;
    }
    if (j.tree.depth + 1 > (uint32_t)SB_STACK) {
        why = "scene BVH deeper than the traversal stack";
        return cudaSuccess;
    }
    const uint32_t n = j.n;
    const size_t nq = j.tree.nodes.size() / 4;  // uint4 count
    cudaError_t e = grow_dev(nodes, nodeCap, nq ? nq : 4);
    if (e == cudaSuccess) e = grow_dev(items, itemCap, n ? n : 1);
    if (e == cudaSuccess && nq)
        e = cudaMemcpy(nodes, j.tree.nodes.data(), j.tree.nodes.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n)
        e = cudaMemcpy(items, j.tree.items.data(), j.tree.items.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    wideReady = false;
    if (j.wide && n && j.wideOk && j.wt.depth + 1 <= (uint32_t)SB_STACK) {
        const size_t wq = j.wt.nodes.size() / 4;
        e = grow_dev(wnodes, wnodeCap, wq);
        if (e == cudaSuccess) e = grow_dev(witems, witemCap, n);
        if (e == cudaSuccess) e = cudaMemcpy(wnodes, j.wt.nodes.data(), j.wt.nodes.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(witems, j.wt.items.data(), j.wt.items.size() * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        wideReady = true;
        wideCount = (uint32_t)(j.wt.nodes.size() / flat::WIDE_WORDS);
        wideDepth = j.wt.depth;
    }
    root = j.tree.root;
    depth = j.tree.depth;
    itemCount = n;
    slotRoot = std::move(j.slotRoot);
    slotEnd = std::move(j.slotEnd);
    srcToSlot = std::move(j.srcToSlot);
    skip.assign(j.slots, 0);
    dyn.clear();
    ready = true;
    overflowed = false;
    // slots that moved or were refit while a background build ran
    for (uint32_t s : j.movedList) mark_slot(s);
    if (j.movedOverflow) overflowed = true;
    marksDirty = true;
    ++builds;
    lastBuildMs = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - j.t0).count();
    return cudaSuccess;
}

cudaError_t FlatScene::finish(cudaStream_t st, std::string& why) {
    if (!job) return cudaSuccess;
    if (job->th.joinable()) job->th.join();
    std::unique_ptr<Job> j = std::move(job);
    // a structural change since its inputs were read: dropped (dirty stays set)
    return j->generation == generation ? install(*j, st, why) : cudaSuccess;
}

cudaError_t FlatScene::prepare(const SceneBuffers& B, const uint32_t* order, uint32_t orderCount, cudaStream_t st,
                               std::string& why) {
    if (!enabled) {
        ready = false;
        return cudaSuccess;
    }
    // a finished build is installed; in blocking mode (switched back while a
    // build ran) the trace waits for it
    if (job && (!background || job->done.load(std::memory_order_acquire))) {
        cudaError_t e = finish(st, why);
        if (e != cudaSuccess) return e;
    }
    if (dirty && !job) {
        std::unique_ptr<Job> j(new Job());
        cudaError_t e = snapshot(B, order, orderCount, st, *j);
        if (e != cudaSuccess) return e;
        dirty = false;
        ready = false;  // the old tree no longer describes the scene
        if (background) {
            Job* jp = j.get();
            job = std::move(j);
            jp->th = std::thread([jp] {
                compute(*jp);
                jp->done.store(true, std::memory_order_release);
            });
        } else {
            compute(*j);
            e = install(*j, st, why);
            if (e != cudaSuccess) return e;
        }
    }
    if (ready && marksDirty) {
        cudaError_t e = grow_dev(dSkip, skipCap, skip.size() ? skip.size() : 1);
        if (e == cudaSuccess) e = grow_dev(dDyn, dynCap, kMaxDynamic);
        if (e == cudaSuccess && !skip.empty())
            e = cudaMemcpyAsync(dSkip, skip.data(), skip.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !dyn.empty())
            e = cudaMemcpyAsync(dDyn, dyn.data(), dyn.size() * 4, cudaMemcpyHostToDevice, st);
        // pageable sources: wait so the vectors may change after return
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        marksDirty = false;
    }
    return cudaSuccess;
}

void FlatScene::mark_slot(uint32_t s) {
    if (job) {  // a background build runs: its tree will not cover this slot's new state
        Job& j = *job;
        if (s >= j.moved.size() || j.moved[s]) return;
        if (j.movedList.size() >= kMaxDynamic) {
            j.movedOverflow = true;
            return;
        }
        j.moved[s] = 1;
        j.movedList.push_back(s);
        return;
    }
    if (!ready || dirty || s >= skip.size() || skip[s]) return;
    if (dyn.size() >= kMaxDynamic) {
        overflowed = true;  // the two-level walk takes over until the next rebuild
        return;
    }
    skip[s] = 1;
    dyn.push_back(s);
    marksDirty = true;
}

void FlatScene::mark_source(uint32_t src) {
    const std::vector<uint32_t>& m = job ? job->srcToSlot : srcToSlot;
    if (src < m.size()) mark_slot(m[src]);
}

void FlatScene::mark_blas_range(uint32_t r0, uint32_t r1) {
    const std::vector<uint32_t>& lo = job ? job->slotRoot : slotRoot;
    const std::vector<uint32_t>& hi = job ? job->slotEnd : slotEnd;
    for (uint32_t s = 0; s < lo.size(); ++s)
        if (lo[s] < r1 && r0 < hi[s]) mark_slot(s);
}

void FlatScene::fill(DevScene& S) const {
    const bool on = enabled && ready && !overflowed;
    S.flatOn = on ? 1 : 0;
    S.flatNodes = on ? nodes : nullptr;
    S.flatItems = on ? items : nullptr;
    S.wideNodes = on && wide && wideReady ? wnodes : nullptr;
    S.wideItems = on && wide && wideReady ? witems : nullptr;
    S.wideNodeCount = on && wide && wideReady ? wideCount : 0u;
    S.wideDepth = on && wide && wideReady ? wideDepth : 0u;
    S.flatRoot = on ? root : flat::ENTRY_NONE;
    S.slotSkip = on ? dSkip : nullptr;
    S.dynList = on ? dDyn : nullptr;
    S.dynCount = on ? (uint32_t)dyn.size() : 0u;
}

void FlatScene::release() {
    if (job) {  // a background build still runs: wait for it and drop it
        if (job->th.joinable()) job->th.join();
        job.reset();
    }
    if (nodes) cudaFree(nodes);
    if (items) cudaFree(items);
    if (dSkip) cudaFree(dSkip);
    if (dDyn) cudaFree(dDyn);
    if (wnodes) cudaFree(wnodes);
    if (witems) cudaFree(witems);
    wnodes = nullptr;
    witems = nullptr;
    wnodeCap = witemCap = 0;
    wideReady = false;
    nodes = nullptr;
    items = nullptr;
    dSkip = nullptr;
    dDyn = nullptr;
    nodeCap = itemCap = skipCap = dynCap = 0;
    ready = false;
    dirty = true;
}

}  // namespace sb
