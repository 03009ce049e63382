// Host-only check of the product BVH builder (jarabotransientrendering_b200/csrc/bvh_build.cpp):
// reads vertices/triangles from a raw file, builds, and verifies the invariants the GPU
// traversal relies on: every triangle appears exactly once in leaf order, child boxes contain
// their triangles, leaf refs and child indices are in range, every node is reachable, the
// four-child depth is what was reported and the reported stack covers it.
// Usage: bvh_check FILE  (FILE: u32 nv, u32 nt, float[nv*3], u32[nt*3])
#include <cstdio>
#include <cstring>
#include <vector>
#include "bvh_build.h"

int main(int argc, char** argv) {
    FILE* f = std::fopen(argv[1], "rb");
    uint32_t nv, nt;
    if (!f || std::fread(&nv, 4, 1, f) != 1 || std::fread(&nt, 4, 1, f) != 1) return 2;
    std::vector<float> v(3 * (size_t)nv);
    std::vector<uint32_t> t(3 * (size_t)nt);
    if (std::fread(v.data(), 4, v.size(), f) != v.size() || std::fread(t.data(), 4, t.size(), f) != t.size()) return 2;
    std::fclose(f);
    trh::BvhBuildResult r;
    std::string msg;
    if (!trh::build_bvh(v.data(), nv, t.data(), nt, 4, r, &msg)) { std::printf("build failed: %s\n", msg.c_str()); return 1; }
    std::vector<int> seen(nt, 0);
    for (const trh::GpuTri& g : r.tris) {
        if (g.id >= nt) { std::printf("bad id\n"); return 1; }
        seen[g.id]++;
        const float* p[3] = {&v[3 * (size_t)t[3 * (size_t)g.id]], &v[3 * (size_t)t[3 * (size_t)g.id + 1]], &v[3 * (size_t)t[3 * (size_t)g.id + 2]]};
        if (std::memcmp(g.v0, p[0], 12) || std::memcmp(g.v1, p[1], 12) || std::memcmp(g.v2, p[2], 12)) { std::printf("vertex mismatch\n"); return 1; }
    }
    for (uint32_t i = 0; i < nt; ++i) if (seen[i] != 1) { std::printf("triangle %u seen %d times\n", i, seen[i]); return 1; }
    // walk the tree: every leaf triangle lies inside the box its parent stores for that child
    struct Item { int32_t node; uint32_t depth; };
    std::vector<Item> st{{0, 0}};
    uint32_t maxd = 0, leaves = 0, visited = 0;
    while (!st.empty()) {
        Item it = st.back(); st.pop_back();
        if (it.node < 0 || (size_t)it.node >= r.nodes.size()) { std::printf("bad node\n"); return 1; }
        ++visited;
        const trh::GpuNode& n = r.nodes[it.node];
        if (it.depth + 1 > maxd) maxd = it.depth + 1;          // four-child levels (root = 1)
        for (int c = 0; c < 4; ++c) {
            float lo[3] = {n.lox[c], n.loy[c], n.loz[c]};
            float hi[3] = {n.hix[c], n.hiy[c], n.hiz[c]};
            int32_t ref = n.child[c];
            if (ref >= 0) { st.push_back({ref, it.depth + 1}); continue; }
            uint32_t u = (uint32_t)(~ref), first = u >> 3, cnt = u & 7u;
            if (cnt == 0) continue;
            ++leaves;
            if (first + cnt > r.tris.size() || cnt > 4) { std::printf("bad leaf\n"); return 1; }
            for (uint32_t k = first; k < first + cnt; ++k) {
                const float* q[3] = {r.tris[k].v0, r.tris[k].v1, r.tris[k].v2};
                for (auto* pt : q) for (int a = 0; a < 3; ++a)
                    if (pt[a] < lo[a] || pt[a] > hi[a]) { std::printf("triangle outside its box\n"); return 1; }
            }
        }
    }
    if (visited != r.nodes.size()) { std::printf("unreachable nodes %u of %zu\n", visited, r.nodes.size()); return 1; }
    std::printf("{\"nodes\": %zu, \"leaves\": %u, \"depth\": %u, \"walk_depth\": %u, \"stack\": %u, "
                "\"binary_depth\": %u, \"build_ms\": %.1f}\n",
                r.nodes.size(), leaves, r.depth, maxd, r.stack, r.binary_depth, r.build_ms);
    // the traversal stack holds at most three siblings per level of the path being walked
    return (maxd != r.depth || r.stack < 3 * maxd) ? 1 : 0;
}
