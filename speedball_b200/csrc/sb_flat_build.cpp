// sb_flat_build.cpp — host builder of the scene BVH: a binned-SAH binary tree
// over (triangle, instance slot) items with world-space bounds, emitted in the
// child-pair layout the traversal reads (sb_flat.h).
//
// This is a derived acceleration structure, built on structural changes only
// (scene upload, instance set, TLAS build), like the reference's CPU-built
// BVHs. The reference's per-instance BLASes and TLAS stay the wire format and
// are still refit and rebuilt bit-exactly; the scene BVH only decides which
// (triangle, instance) pairs a ray tests, and the tests themselves run in the
// instance's local space exactly as the reference's.
#include "sb_flat.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

// The 8-wide tree is collapsed from a binary SAH tree. SB_WIDE_COLLAPSE_SAH 1
// (default): the binary tree has one item per leaf and the SAH-optimal
// dynamic program forms the wide nodes and leaves of up to WIDE_LEAF_MAX items,
// an item test costing SB_WIDE_ITEM_COST wide-node visits; 0: the binary tree
// has leaves of up to WIDE_LEAF_MAX items and each wide node opens the largest
// interior child until eight. On the atrium (CPU walk of 200,000 rays over the
// triangles' boxes) the program gives 6.46 against 6.73 node visits and 1.80
// against 1.91 item tests per ray, 7.2 against 4.3 children per node.
#ifndef SB_WIDE_COLLAPSE_SAH
#define SB_WIDE_COLLAPSE_SAH 1
#endif
#ifndef SB_WIDE_BINARY_LEAF
#define SB_WIDE_BINARY_LEAF (SB_WIDE_COLLAPSE_SAH ? 1u : WIDE_LEAF_MAX)
#endif
#ifndef SB_WIDE_ITEM_COST
#define SB_WIDE_ITEM_COST 0.5f
#endif

namespace sb {
namespace flat {

namespace {

constexpr int BINS = 16;

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    float area() const {
        float d[3];
        for (int a = 0; a < 3; ++a) d[a] = hi[a] - lo[a];
        if (d[0] < 0.f) return 0.f;
        return 2.f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

// Tree nodes under construction (interior: count == 0).
struct Nodes {
    std::vector<Box> box;
    std::vector<uint32_t> left, right, first, count;
    uint32_t make() {
        box.emplace_back();
        left.push_back(0);
        right.push_back(0);
        first.push_back(0);
        count.push_back(0);
        return (uint32_t)box.size() - 1;
    }
    size_t size() const { return box.size(); }
};

struct Bins {
    Box bb[3][BINS];
    uint32_t bc[3][BINS] = {};
    void merge(const Bins& o) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < BINS; ++b) {
                bb[a][b].grow(o.bb[a][b]);
                bc[a][b] += o.bc[a][b];
            }
    }
};

// Items of a leaf range by instance slot, stable (equal slots keep their
// order): insertion sort in place for the small ranges leaves have (a library
// stable sort allocates a buffer per call), the library's above that.
template <class It>
void sort_by_slot(It first, It last, const uint32_t* itemSlot) {
    if (last - first > 32) {
        std::stable_sort(first, last, [&](uint32_t a, uint32_t b) { return itemSlot[a] < itemSlot[b]; });
        return;
    }
    for (It i = first + 1; i < last; ++i) {
        const uint32_t x = *i;
        It j = i;
        for (; j > first && itemSlot[x] < itemSlot[*(j - 1)]; --j) *j = *(j - 1);
        *j = x;
    }
}

// Runs f(lo, hi, part) over `parts` contiguous pieces of [lo, hi) in parallel.
template <class F> void parallel_ranges(uint32_t lo, uint32_t hi, int parts, F&& f) {
    if (parts <= 1) {
        f(lo, hi, 0);
        return;
    }
    std::vector<std::thread> ts;
    const uint32_t n = hi - lo;
    for (int p = 0; p < parts; ++p) {
        const uint32_t a = lo + (uint32_t)((uint64_t)n * p / parts), b = lo + (uint32_t)((uint64_t)n * (p + 1) / parts);
        ts.emplace_back([&f, a, b, p] { f(a, b, p); });
    }
    for (auto& t : ts) t.join();
}

// One item as the builder moves it: its box, centroid and input index. The
// items themselves are partitioned (not an index array), so every pass over a
// node's range reads memory in order.
struct Prim {
    float lo[3], hi[3], c[3];
    uint32_t id;
};

struct Builder {
    uint32_t maxLeaf = 4;
    std::vector<Prim> prims;
    std::vector<uint32_t> order;  // filled after build: order[k] = prims[k].id
    Nodes N;

    void init(const float* boxes, uint32_t n) {
        prims.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            Prim& p = prims[i];
            std::memcpy(p.lo, boxes + 6 * (size_t)i, 12);
            std::memcpy(p.hi, boxes + 6 * (size_t)i + 3, 12);
            for (int a = 0; a < 3; ++a) p.c[a] = 0.5f * (p.lo[a] + p.hi[a]);
            p.id = i;
        }
    }

    static void grow(Box& b, const Prim& p) {
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = std::min(b.lo[a], p.lo[a]);
            b.hi[a] = std::max(b.hi[a], p.hi[a]);
        }
    }

    // Node box and centroid box of [lo, hi) (parallel over `parts`, at most 64).
    void bounds(uint32_t lo, uint32_t hi, int parts, Box& nb, Box& cb) const {
        Box pn[64], pc[64];
        parallel_ranges(lo, hi, parts, [&](uint32_t a, uint32_t b, int p) {
            Box bn, bc;
            for (uint32_t k = a; k < b; ++k) {
                grow(bn, prims[k]);
                bc.grow(prims[k].c);
            }
            pn[p] = bn;
            pc[p] = bc;
        });
        for (int p = 0; p < parts; ++p) {
            nb.grow(pn[p]);
            cb.grow(pc[p]);
        }
    }

    // Stable partition of [lo, hi) by `left` over `parts` threads: each piece
    // counts its left items, then every piece scatters its items to their
    // places in a scratch copy, which goes back in place. Returns the split.
    std::vector<Prim> scratch;
    template <class Pred>
    uint32_t partition_parallel(uint32_t lo, uint32_t hi, int parts, Pred&& left) {
        std::vector<uint32_t> nl(parts), at(parts), ar(parts);
        parallel_ranges(lo, hi, parts, [&](uint32_t a, uint32_t b, int p) {
            uint32_t c = 0;
            for (uint32_t k = a; k < b; ++k) c += left(prims[k]) ? 1u : 0u;
            nl[p] = c;
        });
        uint32_t totalL = 0;
        for (int p = 0; p < parts; ++p) totalL += nl[p];
        uint32_t l = 0, r = totalL;
        for (int p = 0; p < parts; ++p) {
            const uint32_t a = lo + (uint32_t)((uint64_t)(hi - lo) * p / parts);
            const uint32_t b = lo + (uint32_t)((uint64_t)(hi - lo) * (p + 1) / parts);
            at[p] = l;
            ar[p] = r;
            l += nl[p];
            r += (b - a) - nl[p];
        }
        if (scratch.size() < hi - lo) scratch.resize(hi - lo);
        parallel_ranges(lo, hi, parts, [&](uint32_t a, uint32_t b, int p) {
            uint32_t il = at[p], ir = ar[p];
            for (uint32_t k = a; k < b; ++k) scratch[left(prims[k]) ? il++ : ir++] = prims[k];
        });
        parallel_ranges(lo, hi, parts, [&](uint32_t a, uint32_t b, int) {
            std::memcpy(&prims[a], &scratch[a - lo], (size_t)(b - a) * sizeof(Prim));
        });
        return lo + totalL;
    }

    // Splits [lo, hi) by binned SAH over all three axes at once; returns the
    // split point, or hi for a leaf. `nb` receives the node box.
    uint32_t split(uint32_t lo, uint32_t hi, Box& nb, int parts) {
        const uint32_t n = hi - lo;
        Box cb;
        bounds(lo, hi, parts, nb, cb);
        if (n <= 1) return hi;
        float scale[3];
        for (int a = 0; a < 3; ++a) scale[a] = cb.hi[a] > cb.lo[a] ? BINS / (cb.hi[a] - cb.lo[a]) : 0.0f;
        auto bin_of = [&](const Prim& p, int a) {
            return std::min(BINS - 1, (int)((p.c[a] - cb.lo[a]) * scale[a]));
        };
        Bins local;
        std::vector<Bins> pb(parts > 1 ? parts : 0);
        parallel_ranges(lo, hi, parts, [&](uint32_t a0, uint32_t b0, int p) {
            Bins& B = parts > 1 ? pb[p] : local;
            for (uint32_t k = a0; k < b0; ++k) {
                const Prim& q = prims[k];
                for (int a = 0; a < 3; ++a) {
                    if (scale[a] == 0.0f) continue;
                    const int b = bin_of(q, a);
                    grow(B.bb[a][b], q);
                    ++B.bc[a][b];
                }
            }
        });
        if (parts > 1) {
            local = pb[0];
            for (int p = 1; p < parts; ++p) local.merge(pb[p]);
        }
        const Bins& B = local;
        float best = INFINITY;
        int bestAxis = -1, bestBin = 0;
        for (int a = 0; a < 3; ++a) {
            if (scale[a] == 0.0f) continue;
            float la[BINS];
            uint32_t lc[BINS];
            Box L;
            uint32_t ln = 0;
            for (int b = 0; b < BINS - 1; ++b) {
                L.grow(B.bb[a][b]);
                ln += B.bc[a][b];
                la[b] = L.area();
                lc[b] = ln;
            }
            Box R;
            uint32_t rn = 0;
            for (int b = BINS - 1; b > 0; --b) {
                R.grow(B.bb[a][b]);
                rn += B.bc[a][b];
                if (lc[b - 1] == 0 || rn == 0) continue;
                const float cost = la[b - 1] * lc[b - 1] + R.area() * rn;
                if (cost < best) {
                    best = cost;
                    bestAxis = a;
                    bestBin = b;
                }
            }
        }
        // SAH: traversal step ~ one item test; stop when splitting costs more
        const float leafCost = nb.area() * n;
        if (n <= maxLeaf && (bestAxis < 0 || best + nb.area() >= leafCost)) return hi;
        uint32_t mid = lo + n / 2;
        if (bestAxis >= 0) {
            auto left = [&](const Prim& q) { return bin_of(q, bestAxis) < bestBin; };
            if (parts > 1) {
                mid = partition_parallel(lo, hi, parts, left);
            } else {
                auto it = std::partition(prims.begin() + lo, prims.begin() + hi, left);
                mid = (uint32_t)(it - prims.begin());
            }
        }
        if (mid == lo || mid == hi) mid = lo + n / 2;  // coincident centroids: split by index
        return mid;
    }

    // The subtree of [lo, hi) into T, rooted at T's node `root`.
    void build_subtree(Nodes& T, uint32_t root, uint32_t lo, uint32_t hi) {
        struct Task { uint32_t lo, hi, node; };
        std::vector<Task> st{{lo, hi, root}};
        while (!st.empty()) {
            const Task t = st.back();
            st.pop_back();
            Box nb;
            const uint32_t mid = split(t.lo, t.hi, nb, 1);
            T.box[t.node] = nb;
            if (mid >= t.hi) {
                T.first[t.node] = t.lo;
                T.count[t.node] = t.hi - t.lo;
                continue;
            }
            const uint32_t l = T.make(), r = T.make();
            T.left[t.node] = l;
            T.right[t.node] = r;
            st.push_back({mid, t.hi, r});
            st.push_back({t.lo, mid, l});
        }
    }

    // Large trees: the top splits run one at a time with parallel binning until
    // there are enough independent ranges, then every range's subtree is built
    // on its own thread and stitched in (node indices renumbered).
    void build(uint32_t n) {
        const int threads = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
        const uint32_t root = N.make();
        if (n < 65536 || threads == 1) {
            build_subtree(N, root, 0, n);
        } else {
            struct Task { uint32_t lo, hi, node; };
            std::vector<Task> pending{{0, n, root}}, ready;
            while (!pending.empty()) {
                size_t big = 0;
                for (size_t k = 1; k < pending.size(); ++k)
                    if (pending[k].hi - pending[k].lo > pending[big].hi - pending[big].lo) big = k;
                const Task t = pending[big];
                if (pending.size() + ready.size() >= (size_t)8 * threads || t.hi - t.lo < 32768) break;
                pending.erase(pending.begin() + (long)big);
                Box nb;
                const int parts = t.hi - t.lo >= 262144 ? threads : 1;
                const uint32_t mid = split(t.lo, t.hi, nb, parts);
                N.box[t.node] = nb;
                if (mid >= t.hi) {
                    N.first[t.node] = t.lo;
                    N.count[t.node] = t.hi - t.lo;
                    continue;
                }
                const uint32_t l = N.make(), r = N.make();
                N.left[t.node] = l;
                N.right[t.node] = r;
                pending.push_back({t.lo, mid, l});
                pending.push_back({mid, t.hi, r});
            }
            ready.insert(ready.end(), pending.begin(), pending.end());
            std::vector<Nodes> sub(ready.size());
            std::atomic<size_t> next{0};
            std::vector<std::thread> ts;
            for (int w = 0; w < threads; ++w)
                ts.emplace_back([&] {
                    for (size_t k; (k = next.fetch_add(1)) < ready.size();) {
                        sub[k].make();
                        build_subtree(sub[k], 0, ready[k].lo, ready[k].hi);
                    }
                });
            for (auto& t : ts) t.join();
            // subtree k's nodes 1.. land at base[k] ..; its node 0 is the task's node
            std::vector<size_t> base(ready.size() + 1);
            base[0] = N.size();
            for (size_t k = 0; k < ready.size(); ++k) base[k + 1] = base[k] + sub[k].size() - 1;
            const size_t total = base[ready.size()];
            N.box.resize(total);
            N.left.resize(total);
            N.right.resize(total);
            N.first.resize(total);
            N.count.resize(total);
            next = 0;
            ts.clear();
            for (int w = 0; w < threads; ++w)
                ts.emplace_back([&] {
                    for (size_t k; (k = next.fetch_add(1)) < ready.size();) {
                        const Nodes& T = sub[k];
                        const uint32_t node = ready[k].node;
                        const size_t b0 = base[k];
                        auto map = [&](uint32_t j) { return j == 0 ? node : (uint32_t)(b0 + j - 1); };
                        for (size_t j = 0; j < T.size(); ++j) {
                            const size_t d = j == 0 ? node : b0 + j - 1;
                            N.box[d] = T.box[j];
                            N.first[d] = T.first[j];
                            N.count[d] = T.count[j];
                            N.left[d] = T.count[j] ? 0u : map(T.left[j]);
                            N.right[d] = T.count[j] ? 0u : map(T.right[j]);
                        }
                    }
                });
            for (auto& t : ts) t.join();
        }
        order.resize(n);
        for (uint32_t k = 0; k < n; ++k) order[k] = prims[k].id;
        prims.clear();
        prims.shrink_to_fit();
    }
};

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace

bool build(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, Tree& out) {
    out = Tree{};
    if (n == 0) {
        out.root = ENTRY_NONE;
        return true;
    }
    if (n >= (1u << 24)) return false;
    Builder B;
    B.init(boxes, n);
    B.build(n);
    // the passes below touch every node or item once, independently: split over threads
    const int parts = n >= 65536 ? (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency())) : 1;

    // leaves: items ordered by slot, so consecutive tests reuse the local ray
    // (leaf ranges are disjoint)
    parallel_ranges(0, (uint32_t)B.N.count.size(), parts, [&](uint32_t a, uint32_t b, int) {
        for (uint32_t v = a; v < b; ++v) {
            if (B.N.count[v] < 2) continue;
            sort_by_slot(B.order.begin() + B.N.first[v], B.order.begin() + B.N.first[v] + B.N.count[v], itemSlot);
        }
    });
    out.items.resize(2 * (size_t)n);
    parallel_ranges(0, n, parts, [&](uint32_t a, uint32_t b, int) {
        for (uint32_t k = a; k < b; ++k) {
            out.items[2 * (size_t)k] = itemTri[B.order[k]];
            out.items[2 * (size_t)k + 1] = itemSlot[B.order[k]];
        }
    });

    // pair nodes: one per interior tree node, numbered in pre-order
    const size_t total = B.N.box.size();
    std::vector<uint32_t> pairIndex(total, ENTRY_NONE);
    std::vector<uint32_t> depth(total, 0);
    uint32_t pairs = 0, maxDepth = 0;
    {
        std::vector<uint32_t> st{0};
        while (!st.empty()) {
            uint32_t v = st.back();
            st.pop_back();
            maxDepth = std::max(maxDepth, depth[v]);
            if (B.N.count[v]) continue;
            pairIndex[v] = pairs++;
            depth[B.N.left[v]] = depth[B.N.right[v]] = depth[v] + 1;
            st.push_back(B.N.right[v]);
            st.push_back(B.N.left[v]);
        }
    }
    auto entry = [&](uint32_t v) -> uint32_t {
        if (B.N.count[v] == 0) return pairIndex[v];
        return ENTRY_LEAF | (B.N.count[v] << 24) | B.N.first[v];
    };
    out.nodes.assign(16 * (size_t)pairs, 0u);
    parallel_ranges(0, (uint32_t)total, parts, [&](uint32_t a0, uint32_t b0, int) {
      for (uint32_t v = a0; v < b0; ++v) {
        if (B.N.count[v]) continue;
        uint32_t* q = out.nodes.data() + 16 * (size_t)pairIndex[v];
        const Box& a = B.N.box[B.N.left[v]];
        const Box& b = B.N.box[B.N.right[v]];
        q[0] = fbits(a.lo[0]); q[1] = fbits(a.hi[0]); q[2] = fbits(a.lo[1]); q[3] = fbits(a.hi[1]);
        q[4] = fbits(b.lo[0]); q[5] = fbits(b.hi[0]); q[6] = fbits(b.lo[1]); q[7] = fbits(b.hi[1]);
        q[8] = fbits(a.lo[2]); q[9] = fbits(a.hi[2]); q[10] = fbits(b.lo[2]); q[11] = fbits(b.hi[2]);
        q[12] = entry(B.N.left[v]);
        q[13] = entry(B.N.right[v]);
      }
    });
    out.root = entry(0);
    out.depth = maxDepth;
    std::memcpy(out.rootBox, B.N.box[0].lo, 12);
    std::memcpy(out.rootBox + 3, B.N.box[0].hi, 12);
    return true;
}

}  // namespace flat
}  // namespace sb

namespace sb {
namespace flat {

namespace {

// Outward-rounded 8-bit grid of one axis: lo + q * 2^e covers [lo, hi] for q
// in 0..255. Returns the biased exponent (e + 127) stored in the node.
int axis_exponent(float lo, float hi) {
    double extent = (double)hi - (double)lo;
    int e = -126;
    if (extent > 0.0) {
        e = (int)std::ceil(std::log2(extent / 255.0));
        while (std::ldexp(255.0, e) < extent) ++e;
        e = std::max(e, -126);
    }
    return std::min(e, 127) + 127;
}

}  // namespace

bool build_wide(const float* boxes, const uint32_t* itemTri, const uint32_t* itemSlot, uint32_t n, WideTree& out) {
    out = WideTree{};
    if (n == 0) return true;
    if (n >= (1u << 24)) return false;
    Builder B;
    B.maxLeaf = SB_WIDE_BINARY_LEAF;
    B.init(boxes, n);
    B.build(n);
    for (size_t v = 0; v < B.N.count.size(); ++v) {
        if (B.N.count[v] < 2) continue;
        sort_by_slot(B.order.begin() + B.N.first[v], B.order.begin() + B.N.first[v] + B.N.count[v], itemSlot);
    }

#if SB_WIDE_COLLAPSE_SAH
    // SAH-optimal collapse (Ylitie, Karras and Laine 2017, "Efficient incoherent
    // ray traversal on GPUs through compressed wide BVHs"): per binary node v and
    // slot budget i = 1..8 the least cost of covering v's subtree with at most i
    // slots of the parent; a slot is a leaf of at most WIDE_LEAF_MAX items (a
    // binary leaf, or an interior node whose subtree is that small) or an
    // interior wide node. Costs: area x 1 per wide node, area x 0.3 per item.
    // The builder numbers every child after its parent, so descending node
    // order visits children before parents.
    const size_t nv = B.N.size();
    std::vector<uint32_t> sFirst(nv), sCount(nv);
    constexpr float C_NODE = 1.0f, C_ITEM = SB_WIDE_ITEM_COST;
    std::vector<std::array<float, 9>> cost(nv);
    std::vector<std::array<uint8_t, 9>> how(nv), splitK(nv);  // how: 0 reuse i-1, 1 leaf, 2 interior, 3 split
    auto dp = [&](uint32_t v) {
        const float A = B.N.box[v].area();
        if (B.N.count[v]) {
            sFirst[v] = B.N.first[v];
            sCount[v] = B.N.count[v];
            for (int i = 1; i <= 8; ++i) { cost[v][i] = A * C_ITEM * (float)sCount[v]; how[v][i] = 1; }
            return;
        }
        const uint32_t L = B.N.left[v], R = B.N.right[v];
        sFirst[v] = std::min(sFirst[L], sFirst[R]);
        sCount[v] = sCount[L] + sCount[R];
        float D[9];
        for (int j = 2; j <= 8; ++j) {
            D[j] = INFINITY;
            for (int k = 1; k < j; ++k) {
                const float c = cost[L][k] + cost[R][j - k];
                if (c < D[j]) { D[j] = c; splitK[v][j] = (uint8_t)k; }
            }
        }
        const float leafC = sCount[v] <= WIDE_LEAF_MAX ? A * C_ITEM * (float)sCount[v] : INFINITY;
        const float intC = A * C_NODE + D[8];
        cost[v][1] = std::min(leafC, intC);
        how[v][1] = leafC <= intC ? 1 : 2;
        for (int i = 2; i <= 8; ++i) {
            if (D[i] < cost[v][i - 1]) { cost[v][i] = D[i]; how[v][i] = 3; }
            else { cost[v][i] = cost[v][i - 1]; how[v][i] = 0; }
        }
    };
    // bottom-up by depth: the nodes of one depth depend only on deeper ones, so
    // each depth runs in parallel (children are numbered after their parents)
    {
        std::vector<uint32_t> dep(nv, 0);
        uint32_t maxDep = 0;
        for (size_t v = 0; v < nv; ++v)
            if (!B.N.count[v]) {
                dep[B.N.left[v]] = dep[B.N.right[v]] = dep[v] + 1;
                maxDep = std::max(maxDep, dep[v] + 1);
            }
        std::vector<uint32_t> at(maxDep + 2, 0), byDep(nv);
        for (size_t v = 0; v < nv; ++v) ++at[dep[v] + 1];
        for (uint32_t d = 0; d <= maxDep; ++d) at[d + 1] += at[d];
        {
            std::vector<uint32_t> fill(at.begin(), at.end() - 1);
            for (size_t v = 0; v < nv; ++v) byDep[fill[dep[v]]++] = (uint32_t)v;
        }
        const unsigned hwd = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        for (uint32_t d = maxDep + 1; d-- > 0;) {
            const uint32_t lo = at[d], hi = at[d + 1];
            if (hi - lo < 16384 || hwd == 1) {
                for (uint32_t k = lo; k < hi; ++k) dp(byDep[k]);
                continue;
            }
            std::atomic<uint32_t> next{lo};
            auto run = [&] {
                for (uint32_t k; (k = next.fetch_add(1024)) < hi;)
                    for (uint32_t j = k; j < std::min(hi, k + 1024); ++j) dp(byDep[j]);
            };
            std::vector<std::thread> ts;
            for (unsigned t = 1; t < hwd; ++t) ts.emplace_back(run);
            run();
            for (auto& t : ts) t.join();
        }
    }
    // the slots covering v's subtree with budget i, left subtree first
    auto gather = [&](uint32_t v0, int i0, uint32_t* kids, int& nk) {
        struct Entry { uint32_t v; int i; };
        Entry st[16];
        int sp = 0;
        st[sp++] = {v0, i0};
        while (sp) {
            const Entry e = st[--sp];
            const uint32_t v = e.v;
            int i = e.i;
            while (i > 1 && how[v][i] == 0) --i;
            if (i == 1 || B.N.count[v]) {
                kids[nk++] = v;
                continue;
            }
            const int k = splitK[v][i];
            st[sp++] = {B.N.right[v], i - k};
            st[sp++] = {B.N.left[v], k};
        }
    };
    // a slot is a leaf when its node is a binary leaf or the collapse chose one
    auto is_leaf_slot = [&](uint32_t v) { return B.N.count[v] != 0 || how[v][1] == 1; };
#else
    auto is_leaf_slot = [&](uint32_t v) { return B.N.count[v] != 0; };
    const std::vector<uint32_t>& sFirst = B.N.first;
    const std::vector<uint32_t>& sCount = B.N.count;
#endif

    // One wide node formed from binary node v: its child set, slot assignment,
    // quantised boxes and slot metadata (all words but the child and item
    // bases), its interior children and its leaf slots in slot order.
    struct Formed {
        uint32_t words[WIDE_WORDS];
        uint32_t interior[8], leaf[8];
        int nInterior, nLeaf;
    };
    auto form = [&](uint32_t tv, Formed& F) {
        uint32_t kids[8];
        int nk = 0;
#if SB_WIDE_COLLAPSE_SAH
        if (is_leaf_slot(tv)) kids[nk++] = tv;  // a small root is one leaf slot
        else {
            const int k = splitK[tv][8];
            gather(B.N.left[tv], k, kids, nk);
            gather(B.N.right[tv], 8 - k, kids, nk);
        }
#else
        // children: open the largest interior child until eight (a leaf root is its own child)
        if (B.N.count[tv]) kids[nk++] = tv;
        else {
            kids[nk++] = B.N.left[tv];
            kids[nk++] = B.N.right[tv];
        }
        while (nk < 8) {
            int best = -1;
            float bestArea = -1.0f;
            for (int k = 0; k < nk; ++k)
                if (B.N.count[kids[k]] == 0 && B.N.box[kids[k]].area() > bestArea) {
                    bestArea = B.N.box[kids[k]].area();
                    best = k;
                }
            if (best < 0) break;
            const uint32_t v = kids[best];
            kids[best] = B.N.left[v];
            kids[nk++] = B.N.right[v];
        }
#endif
        // slots by octant: slot bit a set = the child lies toward +a of the node centre
        Box nb;
        for (int k = 0; k < nk; ++k) nb.grow(B.N.box[kids[k]]);
        float ctr[3];
        for (int a = 0; a < 3; ++a) ctr[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
        // (cost, kid, slot) by increasing cost, ties in generation order
        struct Cand { float cost; int kid, slot; };
        Cand cands[64];
        int nc = 0;
        for (int k = 0; k < nk; ++k) {
            const Box& b = B.N.box[kids[k]];
            for (int s = 0; s < 8; ++s) {
                float c = 0.0f;
                for (int a = 0; a < 3; ++a) {
                    float d = 0.5f * (b.lo[a] + b.hi[a]) - ctr[a];
                    c += (s >> a & 1) ? -d : d;
                }
                cands[nc++] = {c, k, s};
            }
        }
        for (int i = 1; i < nc; ++i) {  // stable insertion sort (at most 64)
            const Cand c = cands[i];
            int j = i;
            for (; j > 0 && c.cost < cands[j - 1].cost; --j) cands[j] = cands[j - 1];
            cands[j] = c;
        }
        int slotKid[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        int kidSlot[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        for (int ci = 0; ci < nc; ++ci) {
            const Cand& c = cands[ci];
            if (slotKid[c.slot] < 0 && kidSlot[c.kid] < 0) {
                slotKid[c.slot] = c.kid;
                kidSlot[c.kid] = c.slot;
            }
        }
        uint32_t* w = F.words;
        std::memset(w, 0, sizeof F.words);
        int ex[3];
        for (int a = 0; a < 3; ++a) ex[a] = axis_exponent(nb.lo[a], nb.hi[a]);
        std::memcpy(w + 0, &nb.lo[0], 4);
        std::memcpy(w + 1, &nb.lo[1], 4);
        std::memcpy(w + 2, &nb.lo[2], 4);
        uint32_t imask = 0, itemOff = 0;
        uint8_t meta[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint8_t q[6][8];
        F.nInterior = F.nLeaf = 0;
        for (int s = 0; s < 8; ++s) {
            for (int a = 0; a < 3; ++a) { q[a][s] = 255; q[3 + a][s] = 0; }  // empty slots
            if (slotKid[s] < 0) continue;
            const uint32_t v = kids[slotKid[s]];
            const Box& b = B.N.box[v];
            for (int a = 0; a < 3; ++a) {
                const double sc = std::ldexp(1.0, ex[a] - 127);
                double lo = std::floor(((double)b.lo[a] - (double)nb.lo[a]) / sc);
                double hi = std::ceil(((double)b.hi[a] - (double)nb.lo[a]) / sc);
                q[a][s] = (uint8_t)std::min(255.0, std::max(0.0, lo));
                q[3 + a][s] = (uint8_t)std::min(255.0, std::max(0.0, hi));
            }
            if (!is_leaf_slot(v)) {
                imask |= 1u << s;
                meta[s] = (uint8_t)((1u << 5) | (24u + s));
                F.interior[F.nInterior++] = v;
            } else {
                const uint32_t cnt = sCount[v];
                // a leaf merged from an interior node: its items in slot order too (its
                // range is its own; the parts of a node split across slots are not sorted)
                if (!B.N.count[v] && cnt > 1)
                    sort_by_slot(B.order.begin() + sFirst[v], B.order.begin() + sFirst[v] + cnt, itemSlot);
                meta[s] = (uint8_t)((((1u << cnt) - 1u) << 5) | itemOff);
                F.leaf[F.nLeaf++] = v;
                itemOff += cnt;
            }
        }
        w[3] = (uint32_t)ex[0] | (uint32_t)ex[1] << 8 | (uint32_t)ex[2] << 16 | imask << 24;
        w[6] = meta[0] | meta[1] << 8 | meta[2] << 16 | (uint32_t)meta[3] << 24;
        w[7] = meta[4] | meta[5] << 8 | meta[6] << 16 | (uint32_t)meta[7] << 24;
        for (int r = 0; r < 6; ++r) {
            w[8 + 2 * r] = q[r][0] | q[r][1] << 8 | q[r][2] << 16 | (uint32_t)q[r][3] << 24;
            w[9 + 2 * r] = q[r][4] | q[r][5] << 8 | q[r][6] << 16 | (uint32_t)q[r][7] << 24;
        }
    };

    // Breadth first, one level at a time: the level's nodes are formed in
    // parallel (forming reads the collapse tables at random, which is memory
    // latency), then numbered in queue order. Each node's interior children take
    // the next node indices and its leaf items the next item positions, so the
    // layout is the one a sequential breadth-first pass gives.
    out.nodes.assign(WIDE_WORDS, 0u);
    std::vector<uint32_t> level{0}, levelW{0};  // binary node and wide index per node of the level
    std::vector<Formed> formed;
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    uint32_t maxDepth = 0;
    for (uint32_t depth = 0; !level.empty(); ++depth) {
        maxDepth = depth;
        formed.resize(level.size());
        const size_t m = level.size();
        const unsigned nth = m >= 4096 ? hw : 1u;
        std::atomic<size_t> next{0};
        auto run = [&] {
            for (size_t i; (i = next.fetch_add(256)) < m;)
                for (size_t k = i; k < std::min(m, i + 256); ++k) form(level[k], formed[k]);
        };
        std::vector<std::thread> ts;
        for (unsigned t = 1; t < nth; ++t) ts.emplace_back(run);
        run();
        for (auto& t : ts) t.join();
        std::vector<uint32_t> nextLevel, nextW;
        for (size_t i = 0; i < m; ++i) {
            const Formed& F = formed[i];
            const uint32_t childBase = (uint32_t)(out.nodes.size() / WIDE_WORDS);
            const uint32_t itemBase = (uint32_t)(out.items.size() / 2);
            for (int k = 0; k < F.nLeaf; ++k) {
                const uint32_t v = F.leaf[k];
                for (uint32_t j = 0; j < sCount[v]; ++j) {
                    out.items.push_back(itemTri[B.order[sFirst[v] + j]]);
                    out.items.push_back(itemSlot[B.order[sFirst[v] + j]]);
                }
            }
            for (int k = 0; k < F.nInterior; ++k) {
                nextLevel.push_back(F.interior[k]);
                nextW.push_back(childBase + (uint32_t)k);
            }
            out.nodes.resize((size_t)(childBase + F.nInterior) * WIDE_WORDS, 0u);
            uint32_t* w = out.nodes.data() + (size_t)levelW[i] * WIDE_WORDS;
            std::memcpy(w, F.words, sizeof F.words);
            w[4] = childBase;
            w[5] = itemBase;
        }
        level.swap(nextLevel);
        levelW.swap(nextW);
    }
    out.depth = maxDepth;
    return true;
}

}  // namespace flat
}  // namespace sb
