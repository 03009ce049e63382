// bvh_build.cpp - binned-SAH BVH builder (host) producing the 64-byte two-child node layout
// the GPU traversal reads.  Replaces Embree's BVH build inside World::freeze / rtcCommit
// (src/RayTracing/World.h:543-550) for the GPU path.
#include "bvh_build.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
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

// Builder::build fills BinNodes (no initialisers: the array is allocated for all node slots and
// only the used ones are written).
using Node = BinNode;
inline Box box_of(const BinNode& n) {
    Box b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = n.lo[k]; b.hi[k] = n.hi[k]; }
    return b;
}
inline void set_box(BinNode& n, const Box& b) {
    for (int k = 0; k < 3; ++k) { n.lo[k] = b.lo[k]; n.hi[k] = b.hi[k]; }
}

constexpr int kBins = 32;

// Subtrees larger than this are built on their own thread (up to the hardware's thread count);
// nodes larger than kParallelBinning bin their triangles on several threads.
constexpr uint32_t kParallelCutoff = 16384;
constexpr uint32_t kParallelBinning = 1u << 16;
// nodes of at most kSmall triangles evaluate the SAH candidates without bins
constexpr uint32_t kSmall = 16;
static_assert(kBins <= 32, "occupied-bin masks are 32 bits");

// Triangle bounds and centroid bounds of a range plus, per axis, the bins of the centroids
// (bin boxes and counts).  Built by one pass over the range; partial results merge exactly
// (min / max and counts), so the split chosen does not depend on how the range was divided.
struct Binning {
    Box nb, cb;
    Box bb[3][kBins];
    uint32_t bc[3][kBins];
    void clear() {
        nb.empty(); cb.empty();
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < kBins; ++b) { bb[a][b].empty(); bc[a][b] = 0; }
    }
    void merge(const Binning& o) {
        nb.grow(o.nb); cb.grow(o.cb);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < kBins; ++b) { bb[a][b].grow(o.bb[a][b]); bc[a][b] += o.bc[a][b]; }
    }
};

// a triangle as the builder moves it: bounds, centroid, id (partitioned in place, so every
// pass over a node's range reads memory sequentially)
struct Prim { Box b; float c[3]; uint32_t id; };

struct Builder {
    Prim* prim;
    std::unique_ptr<Node[]> nodes;    // Builder::capacity(nt) slots handed out by `take`
    std::atomic<uint32_t> next{0};
    std::atomic<uint32_t> depth{0};
    std::atomic<int> threads{1};
    int max_threads = 1;
    uint32_t max_leaf;

    static int bin_of(float c, float lo, float scale) {
        int b = (int)((c - lo) * scale);
        return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
    }

    // node and centroid bounds of [first, first + count)
    void bounds(uint32_t first, uint32_t count, Box& nb, Box& cb) const {
        nb.empty(); cb.empty();
        for (uint32_t i = first; i < first + count; ++i) {
            nb.grow(prim[i].b);
            cb.growp(prim[i].c);
        }
    }
    // bins of [first, first + count) over the centroid box cb
    void bin_range(uint32_t first, uint32_t count, const Box& cb, Binning& B) const {
        float scale[3];
        for (int a = 0; a < 3; ++a) {
            const float ext = cb.hi[a] - cb.lo[a];
            scale[a] = ext > 0.f ? (float)kBins / ext : 0.f;
        }
        for (uint32_t i = first; i < first + count; ++i) {
            const Prim& q = prim[i];
            for (int a = 0; a < 3; ++a) {
                if (!(scale[a] > 0.f)) continue;
                const int b = bin_of(q.c[a], cb.lo[a], scale[a]);
                B.bb[a][b].grow(q.b);
                B.bc[a][b]++;
            }
        }
    }
    // the same two passes split over `nt` threads
    void bin_parallel(uint32_t first, uint32_t count, Binning& B, int nt) const {
        std::vector<Binning> part((size_t)nt);
        std::vector<std::thread> th;
        const uint32_t chunk = (count + (uint32_t)nt - 1) / (uint32_t)nt;
        auto run = [&](auto&& f) {
            th.clear();
            for (int k = 0; k < nt; ++k) {
                const uint32_t a = first + (uint32_t)k * chunk;
                const uint32_t n = a >= first + count ? 0u : std::min(chunk, first + count - a);
                th.emplace_back([&, k, a, n] { f(k, a, n); });
            }
            for (auto& t : th) t.join();
        };
        run([&](int k, uint32_t a, uint32_t n) { part[k].clear(); bounds(a, n, part[k].nb, part[k].cb); });
        B.clear();
        for (int k = 0; k < nt; ++k) { B.nb.grow(part[k].nb); B.cb.grow(part[k].cb); }
        const Box cb = B.cb;
        run([&](int k, uint32_t a, uint32_t n) { bin_range(a, n, cb, part[k]); });
        for (int k = 0; k < nt; ++k)
            for (int ax = 0; ax < 3; ++ax)
                for (int b = 0; b < kBins; ++b) { B.bb[ax][b].grow(part[k].bb[ax][b]); B.bc[ax][b] += part[k].bc[ax][b]; }
    }

    // Node slots are handed out in chunks of kChunk per thread, so threads write disjoint parts
    // of the node array (no false sharing, one atomic per chunk).
    static constexpr uint32_t kChunk = 1024;
    struct Slots { uint32_t cur = 0, end = 0; };
    uint32_t take(Slots& sl) {
        if (sl.cur == sl.end) {
            sl.cur = next.fetch_add(kChunk, std::memory_order_relaxed);
            sl.end = sl.cur + kChunk;
        }
        return sl.cur++;
    }
    static size_t capacity(uint32_t nt) {
        // 2 nt - 1 nodes, plus one partly used chunk per thread (at most one thread per node
        // of more than kParallelCutoff triangles, and the first)
        return 2 * (size_t)nt + (size_t)kChunk * (2 * (size_t)nt / kParallelCutoff + 3);
    }

    // Splits [first, first + count) so the triangles whose centroid bin on `ax` is <= split
    // come first; returns the boundary and the triangle and centroid bounds of both sides.
    uint32_t partition(uint32_t first, uint32_t count, int ax, float lo, float scale, int split, Box bx[2],
                       Box cx[2]) const {
        bx[0].empty(); bx[1].empty(); cx[0].empty(); cx[1].empty();
        uint32_t i = first, j = first + count;
        while (true) {
            while (i < j && bin_of(prim[i].c[ax], lo, scale) <= split) {
                bx[0].grow(prim[i].b); cx[0].growp(prim[i].c); ++i;
            }
            while (i < j && bin_of(prim[j - 1].c[ax], lo, scale) > split) {
                --j; bx[1].grow(prim[j].b); cx[1].growp(prim[j].c);
            }
            if (i >= j) break;
            std::swap(prim[i], prim[j - 1]);
        }
        return i;
    }

    uint32_t build(uint32_t first, uint32_t count, uint32_t d) {
        Slots sl;
        return build(first, count, d, sl, nullptr, nullptr);
    }
    // nb0 / cb0: the range's triangle and centroid bounds when the parent already has them
    uint32_t build(uint32_t first, uint32_t count, uint32_t d, Slots& sl, const Box* nb0, const Box* cb0) {
        const uint32_t me = take(sl);
        Node& nd = nodes[me];
        nd.left = nd.right = -1;
        nd.first = 0; nd.count = 0;
        uint32_t dd = depth.load(std::memory_order_relaxed);
        while (d > dd && !depth.compare_exchange_weak(dd, d)) {}
        Binning B;
        const bool wide = count >= kParallelBinning && max_threads > 1;
        if (wide) {
            bin_parallel(first, count, B, std::min(max_threads, 16));
        } else {
            B.clear();
            if (nb0) { B.nb = *nb0; B.cb = *cb0; }
            else bounds(first, count, B.nb, B.cb);
        }
        const Box& nb = B.nb;
        const Box& cb = B.cb;
        set_box(nd, nb);
        auto make_leaf = [&]() {
            nd.first = first; nd.count = count;
            nd.n_tris = count;
            return me;
        };
        // SAH leaf test: keep as a leaf when small enough
        if (count <= max_leaf && count <= 2) return make_leaf();
        float best = 3.4e38f; int bax = -1, bsplit = -1;
        if (count <= kSmall) {
            // the same candidates as the binned sweep below, evaluated directly: a split after
            // each occupied bin but the last (splits between two occupied bins all give that
            // cost, and the sweep keeps the first), axes and bins in the same order
            for (int ax = 0; ax < 3; ++ax) {
                const float ext = cb.hi[ax] - cb.lo[ax];
                if (!(ext > 0.f)) continue;
                const float scale = (float)kBins / ext;
                int bins[kSmall];
                uint32_t occupied = 0;                    // bit mask of occupied bins
                for (uint32_t i = 0; i < count; ++i) {
                    bins[i] = bin_of(prim[first + i].c[ax], cb.lo[ax], scale);
                    occupied |= 1u << bins[i];
                }
                const int top = 31 - __builtin_clz(occupied);
                for (uint32_t m = occupied & ~(1u << top); m; m &= m - 1) {
                    const int v = __builtin_ctz(m);
                    Box lbox, rbox; lbox.empty(); rbox.empty();
                    uint32_t nl = 0, nr = 0;
                    for (uint32_t i = 0; i < count; ++i) {
                        if (bins[i] <= v) { lbox.grow(prim[first + i].b); ++nl; }
                        else { rbox.grow(prim[first + i].b); ++nr; }
                    }
                    const float cost = lbox.area() * (float)nl + rbox.area() * (float)nr;
                    if (cost < best) { best = cost; bax = ax; bsplit = v; }
                }
            }
        } else {
        if (!wide) bin_range(first, count, cb, B);
        for (int ax = 0; ax < 3; ++ax) {
            const float ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.f)) continue;
            const Box* bb = B.bb[ax];
            const uint32_t* bc = B.bc[ax];
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
        }
        if (count <= max_leaf) {
            // leaf if splitting does not pay (traversal cost ~ 1 triangle test)
            float leaf_cost = nb.area() * (float)count;
            if (bax < 0 || best + nb.area() >= leaf_cost) return make_leaf();
        }
        uint32_t mid;
        Box bx[2], cx[2];
        bool known = false;                 // children's bounds come from the partition
        if (bax < 0) {
            mid = first + count / 2;
        } else {
            float scale = (float)kBins / (cb.hi[bax] - cb.lo[bax]);
            mid = partition(first, count, bax, cb.lo[bax], scale, bsplit, bx, cx);
            known = true;
            if (mid == first || mid == first + count) { mid = first + count / 2; known = false; }
        }
        const Box* lb = known ? &bx[0] : nullptr;
        const Box* lc = known ? &cx[0] : nullptr;
        const Box* rb = known ? &bx[1] : nullptr;
        const Box* rc2 = known ? &cx[1] : nullptr;
        int32_t l, r;
        if (count > kParallelCutoff && threads.fetch_add(1) < max_threads) {
            uint32_t rr = 0;
            std::thread t([&] {
                Slots ts;
                rr = build(mid, first + count - mid, d + 1, ts, rb, rc2);
            });
            l = (int32_t)build(first, mid - first, d + 1, sl, lb, lc);
            t.join();
            threads.fetch_sub(1);
            r = (int32_t)rr;
        } else {
            if (count > kParallelCutoff) threads.fetch_sub(1);
            l = (int32_t)build(first, mid - first, d + 1, sl, lb, lc);
            r = (int32_t)build(mid, first + count - mid, d + 1, sl, rb, rc2);
        }
        nd.left = l; nd.right = r; nd.count = 0;
        nd.n_tris = nodes[l].n_tris + nodes[r].n_tris;
        return me;
    }
};

}  // namespace

bool build_bvh(const float* v, uint32_t nv, const uint32_t* tri, uint32_t nt, uint32_t max_leaf,
               BvhBuildResult& out, std::string* msg, bool write_tris) {
    auto t0 = std::chrono::steady_clock::now();
    if (nt == 0) { if (msg) *msg = "scene has no triangles"; return false; }
    if (nt >= (1u << 28)) { if (msg) *msg = "too many triangles"; return false; }
    if (max_leaf < 1 || max_leaf > 7) max_leaf = 4;
    const int hw = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    // run f(begin, end) over [0, n) on up to hw threads
    auto parallel_for = [&](uint32_t n, auto&& f) {
        const int k = (int)std::min<uint32_t>((uint32_t)hw, std::max(1u, n / 8192u));
        if (k <= 1) { f(0u, n); return; }
        std::vector<std::thread> th;
        const uint32_t chunk = (n + (uint32_t)k - 1) / (uint32_t)k;
        for (int i = 0; i < k; ++i) {
            const uint32_t a = (uint32_t)i * chunk, b = std::min(n, a + chunk);
            if (a < b) th.emplace_back([&f, a, b] { f(a, b); });
        }
        for (auto& t : th) t.join();
    };

    std::unique_ptr<Prim[]> prim(new Prim[nt]);
    std::atomic<int64_t> bad{-1};                // first bad vertex index seen (-1: none)
    std::atomic<int64_t> bad_tri{-1};
    parallel_for(nt, [&](uint32_t a, uint32_t b) {
        for (uint32_t t = a; t < b; ++t) {
            Prim& q = prim[t];
            q.b.empty();
            q.id = t;
            for (int j = 0; j < 3; ++j) {
                const uint32_t vi = tri[3 * (size_t)t + j];
                if (vi >= nv) { bad_tri.store(t); return; }
                const float* p = &v[3 * (size_t)vi];
                if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) { bad.store(vi); return; }
                q.b.growp(p);
            }
            for (int k = 0; k < 3; ++k) q.c[k] = 0.5f * (q.b.lo[k] + q.b.hi[k]);
        }
    });
    if (bad_tri.load() >= 0) {
        // report the first offending triangle of the input (sequential scan)
        for (uint32_t t = 0; t < nt; ++t)
            for (int j = 0; j < 3; ++j)
                if (tri[3 * (size_t)t + j] >= nv) {
                    if (msg) *msg = "triangle " + std::to_string(t) + " references vertex " +
                                    std::to_string(tri[3 * (size_t)t + j]) + " out of range";
                    return false;
                }
    }
    if (bad.load() >= 0) {
        for (uint32_t t = 0; t < nt; ++t)
            for (int j = 0; j < 3; ++j) {
                const uint32_t vi = tri[3 * (size_t)t + j];
                const float* p = &v[3 * (size_t)vi];
                if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {
                    if (msg) *msg = "vertex " + std::to_string(vi) + " is not finite";
                    return false;
                }
            }
    }
    Builder B;
    B.prim = prim.get(); B.max_leaf = max_leaf;
    B.nodes.reset(new Node[Builder::capacity(nt)]);
    B.max_threads = hw;
    B.build(0, nt, 0);

    std::vector<uint32_t> ids(nt);
    parallel_for(nt, [&](uint32_t a, uint32_t b) { for (uint32_t i = a; i < b; ++i) ids[i] = prim[i].id; });
    const bool ok = finish_bvh(B.nodes.get(), Builder::capacity(nt), ids.data(), nt, B.depth.load(), v, tri, write_tris, out);
    out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return ok;
}

// Collapse to four-child nodes: a node starts with its binary children and repeatedly opens the
// interior child of largest surface area (the first on ties) while it has fewer than four.
// Pass 1 records each four-child node's binary children and its subtree's node count and depth;
// pass 2 writes every subtree at its own offsets (depth-first preorder, children in left-to-right
// order, leaf triangles in the same order), large subtrees on their own threads.
bool finish_bvh(const BinNode* nodes, size_t cap, const uint32_t* ids, uint32_t nt, uint32_t binary_depth,
                const float* v, const uint32_t* tri, bool write_tris, BvhBuildResult& out) {
    const int hw = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const Node& root = nodes[0];
    std::unique_ptr<std::array<int32_t, 4>[]> kids(new std::array<int32_t, 4>[cap]);
    std::unique_ptr<uint32_t[]> n4(new uint32_t[cap]);
    std::unique_ptr<uint32_t[]> d4(new uint32_t[cap]);
    std::atomic<int> cthreads{1};
    std::function<void(int32_t)> collapse = [&](int32_t n) {
        int32_t c[4] = {nodes[n].left, nodes[n].right, -1, -1};
        int k = 2;
        while (k < 4) {
            int best = -1;
            float ba = -1.0f;
            for (int j = 0; j < k; ++j) {
                const Node& q = nodes[c[j]];
                if (q.left < 0) continue;
                const float a = box_of(q).area();
                if (a > ba) { ba = a; best = j; }
            }
            if (best < 0) break;
            const Node& q = nodes[c[best]];
            for (int j = k; j > best + 1; --j) c[j] = c[j - 1];
            c[best] = q.left;
            c[best + 1] = q.right;
            ++k;
        }
        kids[n] = {c[0], c[1], c[2], c[3]};
        // the children's subtrees: the largest one of several on another thread
        int32_t sub[4];
        int ns = 0;
        for (int j = 0; j < 4; ++j)
            if (c[j] >= 0 && nodes[c[j]].left >= 0) sub[ns++] = c[j];
        std::thread th;
        int spawned = -1;
        if (ns > 1) {
            int big = 0;
            for (int j = 1; j < ns; ++j)
                if (nodes[sub[j]].n_tris > nodes[sub[big]].n_tris) big = j;
            if (nodes[sub[big]].n_tris > kParallelCutoff && cthreads.fetch_add(1) < hw) {
                spawned = big;
                th = std::thread([&, s0 = sub[big]] { collapse(s0); });
            } else if (nodes[sub[big]].n_tris > kParallelCutoff) {
                cthreads.fetch_sub(1);
            }
        }
        for (int j = 0; j < ns; ++j)
            if (j != spawned) collapse(sub[j]);
        if (spawned >= 0) { th.join(); cthreads.fetch_sub(1); }
        uint32_t cnt = 1, dep = 0;
        for (int j = 0; j < ns; ++j) { cnt += n4[sub[j]]; dep = std::max(dep, d4[sub[j]]); }
        n4[n] = cnt;
        d4[n] = dep + 1;
    };
    std::atomic<uint32_t> leaves{0};
    auto leaf_ref = [&](const Node& n, uint32_t toff) -> int32_t {
        for (uint32_t i = 0; i < n.count; ++i) {
            const uint32_t t = ids[n.first + i];
            out.order[toff + i] = t;
            if (!write_tris) continue;
            GpuTri& g = out.tris[toff + i];
            const uint32_t* ti = &tri[3 * (size_t)t];
            std::memcpy(g.v0, &v[3 * (size_t)ti[0]], 12);
            std::memcpy(g.v1, &v[3 * (size_t)ti[1]], 12);
            std::memcpy(g.v2, &v[3 * (size_t)ti[2]], 12);
            g.id = t; g.pad1 = 0.f; g.pad2 = 0.f;
        }
        leaves.fetch_add(1, std::memory_order_relaxed);
        return ~(int32_t)((toff << 3) | n.count);
    };
    auto write_box = [](GpuNode& g, int j, const Box& bin) {
        // one ulp outward: a ray lying exactly in a face plane of a box (zero direction
        // component, origin on the face) still sees a non-empty slab interval
        Box b = bin;
        for (int k = 0; k < 3; ++k) {
            if (b.lo[k] <= b.hi[k]) {
                b.lo[k] = std::nextafter(b.lo[k], -INFINITY);
                b.hi[k] = std::nextafter(b.hi[k], INFINITY);
            }
        }
        g.lox[j] = b.lo[0]; g.hix[j] = b.hi[0];
        g.loy[j] = b.lo[1]; g.hiy[j] = b.hi[1];
        g.loz[j] = b.lo[2]; g.hiz[j] = b.hi[2];
    };
    auto empty_slot = [](GpuNode& g, int j) {
        g.lox[j] = g.hix[j] = g.loy[j] = g.hiy[j] = g.loz[j] = g.hiz[j] = 0.0f;
        g.child[j] = ~(int32_t)0;             // leaf of 0 triangles: never entered
    };
    std::atomic<int> fthreads{1};
    // four-child node of binary node n at GPU index gi, its leaf triangles from toff
    std::function<void(int32_t, uint32_t, uint32_t)> flat = [&](int32_t n, uint32_t gi, uint32_t toff) {
        GpuNode& g = out.nodes[gi];
        g.pad[0] = g.pad[1] = g.pad[2] = g.pad[3] = 0;
        struct Sub { int32_t n; uint32_t gi, toff; };
        Sub sub[4];
        int ns = 0;
        uint32_t gnext = gi + 1, t = toff;
        for (int j = 0; j < 4; ++j) {
            const int32_t c = kids[n][j];
            if (c < 0) { empty_slot(g, j); continue; }
            const Node& q = nodes[c];
            write_box(g, j, box_of(q));
            if (q.left >= 0) {
                g.child[j] = (int32_t)gnext;
                sub[ns++] = {c, gnext, t};
                gnext += n4[c];
            } else {
                g.child[j] = leaf_ref(q, t);
            }
            t += q.n_tris;
        }
        std::thread th;
        int spawned = -1;
        if (ns > 1) {
            int big = 0;
            for (int j = 1; j < ns; ++j)
                if (nodes[sub[j].n].n_tris > nodes[sub[big].n].n_tris) big = j;
            if (nodes[sub[big].n].n_tris > kParallelCutoff && fthreads.fetch_add(1) < hw) {
                spawned = big;
                th = std::thread([&, sb = sub[big]] { flat(sb.n, sb.gi, sb.toff); });
            } else if (nodes[sub[big].n].n_tris > kParallelCutoff) {
                fthreads.fetch_sub(1);
            }
        }
        for (int j = 0; j < ns; ++j)
            if (j != spawned) flat(sub[j].n, sub[j].gi, sub[j].toff);
        if (spawned >= 0) { th.join(); fthreads.fetch_sub(1); }
    };
    out.order.resize(nt);
    if (write_tris) out.tris.resize(nt);
    else out.tris.clear();
    if (root.left < 0) {
        // single-leaf scene: one node whose first child is the leaf
        out.nodes.assign(1, GpuNode{});
        write_box(out.nodes[0], 0, box_of(root));
        out.nodes[0].child[0] = leaf_ref(root, 0);
        for (int j = 1; j < 4; ++j) empty_slot(out.nodes[0], j);
        out.depth = 1;
    } else {
        collapse(0);
        out.nodes.resize(n4[0]);
        flat(0, 0, 0);
        out.depth = d4[0];
    }
    out.stack = 3 * out.depth + 1;
    out.binary_depth = binary_depth;
    out.leaves = leaves.load();
    return true;
}

}  // namespace trh
