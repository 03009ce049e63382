// bvh_build.cpp - binned-SAH BVH builder (host) producing the 64-byte two-child node layout
// the GPU traversal reads.  Replaces Embree's BVH build inside World::freeze / rtcCommit
// (src/RayTracing/World.h:543-550) for the GPU path.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

namespace trh {
namespace {

struct Box {
    float lo[3], hi[3];
    void empty() { for (int k = 0; k < 3; ++k) { lo[k] = 3.4e38f; hi[k] = -3.4e38f; } }
    void grow(const Box& o) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], o.lo[k]); hi[k] = std::max(hi[k], o.hi[k]); }
    }
    void growp(const float* p) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    float area() const {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx < 0.f) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node { Box box; int32_t left = -1, right = -1; uint32_t first = 0, count = 0; };

constexpr int kBins = 32;

// Subtrees larger than this are built on their own thread (up to the hardware's thread count).
constexpr uint32_t kParallelCutoff = 16384;

struct Builder {
    const Box* tb;
    const float* cen;
    std::vector<uint32_t> idx;
    std::vector<Node> nodes;          // preallocated 2*nt; slots handed out by `next`
    std::atomic<uint32_t> next{0};
    std::atomic<uint32_t> depth{0};
    std::atomic<int> threads{1};
    int max_threads = 1;
    uint32_t max_leaf;

    int bin_of(float c, float lo, float scale) const {
        int b = (int)((c - lo) * scale);
        return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
    }

    uint32_t build(uint32_t first, uint32_t count, uint32_t d) {
        uint32_t me = next.fetch_add(1, std::memory_order_relaxed);
        Box nb, cb; nb.empty(); cb.empty();
        for (uint32_t i = first; i < first + count; ++i) {
            uint32_t t = idx[i];
            nb.grow(tb[t]);
            cb.growp(&cen[3 * t]);
        }
        nodes[me].box = nb;
        uint32_t dd = depth.load(std::memory_order_relaxed);
        while (d > dd && !depth.compare_exchange_weak(dd, d)) {}
        if (count <= max_leaf) {
            // SAH leaf test: keep as a leaf when small enough
            nodes[me].first = first; nodes[me].count = count;
            if (count <= 2) return me;
        }
        float best = 3.4e38f; int bax = -1, bsplit = -1;
        for (int ax = 0; ax < 3; ++ax) {
            float ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.f)) continue;
            float scale = (float)kBins / ext;
            Box bb[kBins]; uint32_t bc[kBins];
            for (int b = 0; b < kBins; ++b) { bb[b].empty(); bc[b] = 0; }
            for (uint32_t i = first; i < first + count; ++i) {
                uint32_t t = idx[i];
                int b = bin_of(cen[3 * t + ax], cb.lo[ax], scale);
                bb[b].grow(tb[t]); bc[b]++;
            }
            float ra[kBins]; uint32_t rc[kBins]; Box acc; acc.empty(); uint32_t n = 0;
            for (int b = kBins - 1; b > 0; --b) { acc.grow(bb[b]); n += bc[b]; ra[b] = acc.area(); rc[b] = n; }
            acc.empty(); n = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bb[b]); n += bc[b];
                if (n == 0 || rc[b + 1] == 0) continue;
                float cost = acc.area() * (float)n + ra[b + 1] * (float)rc[b + 1];
                if (cost < best) { best = cost; bax = ax; bsplit = b; }
            }
        }
        if (count <= max_leaf) {
            // leaf if splitting does not pay (traversal cost ~ 1 triangle test)
            float leaf_cost = nb.area() * (float)count;
            if (bax < 0 || best + nb.area() >= leaf_cost) return me;
        }
        uint32_t mid;
        if (bax < 0) {
            mid = first + count / 2;
        } else {
            float scale = (float)kBins / (cb.hi[bax] - cb.lo[bax]);
            auto it = std::partition(idx.begin() + first, idx.begin() + first + count, [&](uint32_t t) {
                return bin_of(cen[3 * t + bax], cb.lo[bax], scale) <= bsplit;
            });
            mid = (uint32_t)(it - idx.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        }
        int32_t l, r;
        if (count > kParallelCutoff && threads.fetch_add(1) < max_threads) {
            uint32_t rr = 0;
            std::thread t([&] { rr = build(mid, first + count - mid, d + 1); });
            l = (int32_t)build(first, mid - first, d + 1);
            t.join();
            threads.fetch_sub(1);
            r = (int32_t)rr;
        } else {
            if (count > kParallelCutoff) threads.fetch_sub(1);
            l = (int32_t)build(first, mid - first, d + 1);
            r = (int32_t)build(mid, first + count - mid, d + 1);
        }
        nodes[me].left = l; nodes[me].right = r; nodes[me].count = 0;
        return me;
    }
};

}  // namespace

bool build_bvh(const float* v, uint32_t nv, const uint32_t* tri, uint32_t nt, uint32_t max_leaf,
               BvhBuildResult& out, std::string* msg) {
    auto t0 = std::chrono::steady_clock::now();
    if (nt == 0) { if (msg) *msg = "scene has no triangles"; return false; }
    if (max_leaf < 1 || max_leaf > 7) max_leaf = 4;
    std::vector<Box> tb(nt);
    std::vector<float> cen(3 * (size_t)nt);
    for (uint32_t t = 0; t < nt; ++t) {
        tb[t].empty();
        for (int j = 0; j < 3; ++j) {
            uint32_t vi = tri[3 * (size_t)t + j];
            if (vi >= nv) { if (msg) *msg = "triangle " + std::to_string(t) + " references vertex " + std::to_string(vi) + " out of range"; return false; }
            const float* p = &v[3 * (size_t)vi];
            if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {
                if (msg) *msg = "vertex " + std::to_string(vi) + " is not finite";
                return false;
            }
            tb[t].growp(p);
        }
        for (int k = 0; k < 3; ++k) cen[3 * (size_t)t + k] = 0.5f * (tb[t].lo[k] + tb[t].hi[k]);
    }
    Builder B;
    B.tb = tb.data(); B.cen = cen.data(); B.max_leaf = max_leaf;
    B.idx.resize(nt);
    for (uint32_t t = 0; t < nt; ++t) B.idx[t] = t;
    B.nodes.resize(2 * (size_t)nt);
    B.max_threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    B.build(0, nt, 0);
    B.nodes.resize(B.next.load());

    // Flatten: one GpuNode per interior node, depth-first, left child adjacent to its parent.
    out.nodes.clear(); out.tris.clear(); out.leaves = 0;
    out.tris.reserve(nt);
    std::vector<int32_t> gpu_index(B.nodes.size(), -1);
    auto leaf_ref = [&](const Node& n) -> int32_t {
        uint32_t first = (uint32_t)out.tris.size();
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
            uint32_t t = B.idx[i];
            GpuTri g;
            const uint32_t* ti = &tri[3 * (size_t)t];
            std::memcpy(g.v0, &v[3 * (size_t)ti[0]], 12);
            std::memcpy(g.v1, &v[3 * (size_t)ti[1]], 12);
            std::memcpy(g.v2, &v[3 * (size_t)ti[2]], 12);
            g.id = t; g.pad1 = 0.f; g.pad2 = 0.f;
            out.tris.push_back(g);
        }
        out.leaves++;
        return ~(int32_t)((first << 3) | n.count);
    };
    auto write_box = [](GpuNode& g, int slot, const Box& bin) {
        // one ulp outward: a ray lying exactly in a face plane of a box (zero direction
        // component, origin on the face) still sees a non-empty slab interval
        Box b = bin;
        for (int k = 0; k < 3; ++k) {
            if (b.lo[k] <= b.hi[k]) {
                b.lo[k] = std::nextafter(b.lo[k], -INFINITY);
                b.hi[k] = std::nextafter(b.hi[k], INFINITY);
            }
        }
        if (slot == 0) {
            g.a[0] = b.lo[0]; g.a[1] = b.hi[0]; g.a[2] = b.lo[1]; g.a[3] = b.hi[1];
            g.c[0] = b.lo[2]; g.c[1] = b.hi[2];
        } else {
            g.b[0] = b.lo[0]; g.b[1] = b.hi[0]; g.b[2] = b.lo[1]; g.b[3] = b.hi[1];
            g.c[2] = b.lo[2]; g.c[3] = b.hi[2];
        }
    };
    Box emptybox; emptybox.empty();
    if (nt >= (1u << 28)) { if (msg) *msg = "too many triangles"; return false; }
    const Node& root = B.nodes[0];
    if (root.left < 0) {
        // single-leaf scene: a root whose second child is empty
        GpuNode g{};
        out.nodes.push_back(g);
        write_box(out.nodes[0], 0, root.box);
        write_box(out.nodes[0], 1, emptybox);
        out.nodes[0].d[0] = leaf_ref(root);
        out.nodes[0].d[1] = ~(int32_t)0;   // empty leaf (count 0)
    } else {
        std::vector<uint32_t> stack;
        stack.push_back(0);
        gpu_index[0] = 0;
        out.nodes.emplace_back();
        while (!stack.empty()) {
            uint32_t ni = stack.back(); stack.pop_back();
            const Node& n = B.nodes[ni];
            int32_t gi = gpu_index[ni];
            int32_t child[2] = {n.left, n.right};
            int32_t refs[2];
            for (int s = 0; s < 2; ++s) {
                const Node& c = B.nodes[child[s]];
                write_box(out.nodes[gi], s, c.box);
                if (c.left < 0) {
                    refs[s] = leaf_ref(c);
                } else {
                    gpu_index[child[s]] = (int32_t)out.nodes.size();
                    out.nodes.emplace_back();
                    refs[s] = gpu_index[child[s]];
                }
            }
            out.nodes[gi].d[0] = refs[0]; out.nodes[gi].d[1] = refs[1];
            out.nodes[gi].d[2] = 0; out.nodes[gi].d[3] = 0;
            // push right first so the left subtree is laid out next
            for (int s = 1; s >= 0; --s)
                if (B.nodes[child[s]].left >= 0) stack.push_back((uint32_t)child[s]);
        }
    }
    out.depth = B.depth.load();
    out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

}  // namespace trh
