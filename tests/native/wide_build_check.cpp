// CPU check of the 8-wide scene-BVH builder (speedball_b200/csrc/sb_flat_build.cpp):
// random triangle boxes with random instance slots; every item appears exactly
// once, inside the dequantised box of its leaf slot, leaves hold 1..3 items of
// non-decreasing slot, interior slots point at nodes whose own box lies inside
// the slot box, and the tree is no deeper than reported. Prints "ok" or the
// first failure; exit status 0 on success.
#include "sb_flat.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

using namespace sb::flat;

static void slot_box(const uint32_t* w, int s, float lo[3], float hi[3]) {
    float p[3];
    std::memcpy(p, w, 12);
    for (int a = 0; a < 3; ++a) {
        const float sc = std::ldexp(1.0f, (int)((w[3] >> (8 * a)) & 255u) - 127);
        lo[a] = p[a] + (float)((w[8 + 2 * a + (s >> 2)] >> (8 * (s & 3))) & 255u) * sc;
        hi[a] = p[a] + (float)((w[8 + 2 * (3 + a) + (s >> 2)] >> (8 * (s & 3))) & 255u) * sc;
    }
}

int main(int argc, char** argv) {
    const uint32_t n = argc > 1 ? (uint32_t)std::atoi(argv[1]) : 50000;
    const uint32_t seed = argc > 2 ? (uint32_t)std::atoi(argv[2]) : 1;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> U(0.0f, 100.0f), S(0.01f, 2.0f);
    std::vector<float> boxes((size_t)n * 6);
    std::vector<uint32_t> tri(n), slot(n);
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            const float c = U(rng), h = S(rng);
            boxes[6 * i + a] = c - h;
            boxes[6 * i + 3 + a] = c + h;
        }
        tri[i] = i;
        slot[i] = rng() % 37u;
    }
    WideTree wt;
    if (!build_wide(boxes.data(), tri.data(), slot.data(), n, wt)) { std::puts("build failed"); return 1; }
    const size_t nodes = wt.nodes.size() / WIDE_WORDS;
    std::vector<int> seen(n, 0);
    std::vector<uint32_t> level(nodes, 0);
    for (size_t i = 0; i < nodes; ++i) {
        const uint32_t* w = wt.nodes.data() + i * WIDE_WORDS;
        const uint32_t imask = w[3] >> 24;
        for (int s = 0; s < 8; ++s) {
            const uint32_t m = ((s < 4 ? w[6] : w[7]) >> (8 * (s & 3))) & 255u;
            if (!m) continue;
            float lo[3], hi[3];
            slot_box(w, s, lo, hi);
            if ((m & 31u) >= 24u) {
                if (!(imask >> s & 1u)) { std::printf("node %zu slot %d: interior meta without imask\n", i, s); return 1; }
                const uint32_t c = w[4] + __builtin_popcount(imask & ((1u << s) - 1u));
                if (c <= i || c >= nodes) { std::printf("node %zu slot %d: child %u out of order\n", i, s, c); return 1; }
                level[c] = level[i] + 1;
                const uint32_t* cw = wt.nodes.data() + (size_t)c * WIDE_WORDS;
                float cp[3];
                std::memcpy(cp, cw, 12);
                for (int a = 0; a < 3; ++a)
                    if (cp[a] < lo[a]) { std::printf("node %u origin outside its slot box\n", c); return 1; }
                continue;
            }
            const uint32_t cnt = __builtin_popcount(m >> 5), off = m & 31u;
            if (cnt < 1 || cnt > WIDE_LEAF_MAX) { std::printf("leaf of %u items\n", cnt); return 1; }
            uint32_t prevSlot = 0;
            for (uint32_t q = 0; q < cnt; ++q) {
                const uint32_t it = wt.items[2 * (w[5] + off + q)], sl = wt.items[2 * (w[5] + off + q) + 1];
                if (it >= n || sl != slot[it]) { std::printf("item %u: wrong slot\n", it); return 1; }
                if (q && sl < prevSlot) { std::printf("leaf items not in slot order\n"); return 1; }
                prevSlot = sl;
                ++seen[it];
                for (int a = 0; a < 3; ++a)
                    if (boxes[6 * it + a] < lo[a] || boxes[6 * it + 3 + a] > hi[a]) {
                        std::printf("item %u outside its leaf slot box (node %zu slot %d)\n", it, i, s);
                        return 1;
                    }
            }
        }
    }
    for (uint32_t i = 0; i < n; ++i)
        if (seen[i] != 1) { std::printf("item %u appears %d times\n", i, seen[i]); return 1; }
    uint32_t deepest = 0;
    for (uint32_t d : level) deepest = d > deepest ? d : deepest;
    if (deepest > wt.depth) { std::printf("depth %u above the reported %u\n", deepest, wt.depth); return 1; }
    std::printf("ok %zu nodes %.2f children per node depth %u\n", nodes,
                (double)(wt.items.size() / 2 + nodes - 1) / (double)nodes, wt.depth);
    return 0;
}
