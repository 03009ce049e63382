// bvh_gpu.cu - binned-SAH BVH build on the device, with the split rules of the host builder
// (bvh_build.cpp: 32 bins over the centroid bounds, the same SAH sweep and leaf tests, median
// split when no axis can be binned), followed by the shared four-child collapse on the host.
// Replaces Embree's BVH build inside World::freeze / rtcCommit (src/RayTracing/World.h:543-550).
//
// Levels over the nodes of more than kSmall triangles: per level, the nodes' triangle and centroid
// bounds, then per-axis bins, then one thread per node picks the split, then the triangles are
// partitioned into the children's ranges.  Nodes of at most kSmall triangles are finished by one
// thread each (direct evaluation of the same split candidates, two-pointer partition, as the
// host builder does).  Min/max are exact in any order, so every split decision is the host's;
// only the median fallback (no binnable axis) splits by array order, which may differ.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "tr_internal.h"

namespace trh {
using tri::CudaError;
namespace {

constexpr int kBins = 32;
constexpr uint32_t kSmall = 16;
constexpr float kBig = 3.4e38f;
constexpr uint32_t kChunk = 4096;       // positions per block in the bounds / bin kernels

// float min / max through the integer order of IEEE floats (exact, order independent)
__device__ __forceinline__ void amin(float* a, float v) {
    if (v >= 0.0f) atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}
__device__ __forceinline__ void amax(float* a, float v) {
    if (v >= 0.0f) atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}
// the same in shared memory, skipped when v does not improve the stored value: a stored min
// only decreases, so a value not below it now is not below the final one (exact)
__device__ __forceinline__ void amin_s(float* a, float v) {
    if (v < *reinterpret_cast<volatile float*>(a)) amin(a, v);
}
__device__ __forceinline__ void amax_s(float* a, float v) {
    if (v > *reinterpret_cast<volatile float*>(a)) amax(a, v);
}
__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    const int b = (int)((c - lo) * scale);
    return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}
__device__ __forceinline__ float area(const float* lo, const float* hi) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0.f) return 0.f;
    return 2.f * (dx * dy + dy * dz + dz * dx);
}
__device__ __forceinline__ void box_empty(float* lo, float* hi) {
    for (int k = 0; k < 3; ++k) { lo[k] = kBig; hi[k] = -kBig; }
}
__device__ __forceinline__ void box_grow(float* lo, float* hi, const float* olo, const float* ohi) {
    for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], olo[k]); hi[k] = fmaxf(hi[k], ohi[k]); }
}

struct Dev {
    float4 *plo, *phi, *pc;            // per triangle id: bounds and centroid
    uint32_t* ids[2];                  // per position (ping-pong): triangle id
    int32_t* pn[2];                    // per position: active node of the level, -1 when done
    uint4* act[2];                     // active nodes: first, count, out index, depth
    float *nb, *cb, *bb;               // per active node: bounds, centroid bounds; bins [3][kBins] x 6
    uint32_t* bc;                      // bin counts
    int32_t* d_ax;                     // split axis, -1: median split by position
    int32_t* d_split;                  // last bin of the left child
    uint32_t* d_nl;                    // triangles of the left child
    float* d_scale;                    // kBins / centroid extent on the axis
    int32_t* d_child;                  // [2] next-level active index per child, -1 when small
    uint32_t *lcur, *rcur;
    uint4* small;                      // small nodes: first, count, out index, depth
    BinNode* nodes;
    uint32_t* counters;                // 0 nodes, 1 next active, 2 small, 3 max depth, 4 input error
    uint32_t max_leaf;
};

__global__ void k_prims(const float* __restrict__ v, uint32_t nv, const uint32_t* __restrict__ t, uint32_t nt,
                        Dev d) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        float lo[3] = {kBig, kBig, kBig}, hi[3] = {-kBig, -kBig, -kBig};
        bool bad = false;
        for (int j = 0; j < 3 && !bad; ++j) {
            const uint32_t vi = t[3 * (size_t)i + j];
            if (vi >= nv) { bad = true; break; }
            for (int k = 0; k < 3; ++k) {
                const float p = v[3 * (size_t)vi + k];
                if (!isfinite(p)) bad = true;
                lo[k] = fminf(lo[k], p);
                hi[k] = fmaxf(hi[k], p);
            }
        }
        if (bad) atomicOr(&d.counters[4], 1u);
        d.plo[i] = make_float4(lo[0], lo[1], lo[2], 0.f);
        d.phi[i] = make_float4(hi[0], hi[1], hi[2], 0.f);
        d.pc[i] = make_float4(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2]), 0.f);
        d.ids[0][i] = i;
        d.pn[0][i] = 0;
    }
}

// reset the level's accumulators for na nodes
__global__ void k_clear(Dev d, uint32_t na) {
    const uint32_t nbins = na * 3u * kBins;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbins * 6u; i += gridDim.x * blockDim.x) {
        const float e = (i % 6u) < 3 ? kBig : -kBig;
        d.bb[i] = e;
        if (i < na * 6u) { d.nb[i] = e; d.cb[i] = e; }
        if (i < nbins) d.bc[i] = 0;
        if (i < na) { d.lcur[i] = 0; d.rcur[i] = 0; }
    }
}

// the node every position of [p0, p1) belongs to, or -1 (active ranges are contiguous)
__device__ __forceinline__ int32_t block_node(const int32_t* pn, uint32_t p0, uint32_t p1) {
    const int32_t a = pn[p0], b = pn[p1 - 1];
    return (a >= 0 && a == b) ? a : -1;
}

// triangle and centroid bounds of every active node.  Each thread takes kChunk / 256 contiguous
// positions and keeps their bounds in registers while the node stays the same (a node of the
// level holds more than kSmall positions, so a thread meets at most two), then adds them with
// one set of atomics per node; a block whose positions all belong to one node first reduces
// over each warp and collects in shared memory.  min / max are exact, so the result does not
// depend on the order.
__global__ void __launch_bounds__(256) k_bounds(Dev d, int cur, uint32_t nt) {
    constexpr uint32_t kPer = kChunk / 256;
    __shared__ float s[12];
    const uint32_t p0 = blockIdx.x * kChunk, p1 = min(nt, p0 + kChunk);
    const int32_t* pn = d.pn[cur];
    const int32_t one = block_node(pn, p0, p1);
    if (threadIdx.x < 12) s[threadIdx.x] = (threadIdx.x % 6u) < 3 ? kBig : -kBig;
    __syncthreads();
    float b[12];
    int32_t bn = -1;
    auto reset = [&]() {
#pragma unroll
        for (int k = 0; k < 12; ++k) b[k] = (k % 6) < 3 ? kBig : -kBig;
    };
    auto flush = [&](float* nb, float* cb) {
        amin(nb + 0, b[0]); amin(nb + 1, b[1]); amin(nb + 2, b[2]);
        amax(nb + 3, b[3]); amax(nb + 4, b[4]); amax(nb + 5, b[5]);
        amin(cb + 0, b[6]); amin(cb + 1, b[7]); amin(cb + 2, b[8]);
        amax(cb + 3, b[9]); amax(cb + 4, b[10]); amax(cb + 5, b[11]);
    };
    reset();
    const uint32_t q0 = p0 + threadIdx.x * kPer, q1 = min(p1, q0 + kPer);
    for (uint32_t i = q0; i < q1; ++i) {
        const int32_t n = pn[i];
        if (n < 0) continue;
        if (n != bn) {
            if (bn >= 0 && one < 0) flush(d.nb + 6 * bn, d.cb + 6 * bn);
            if (one < 0) reset();
            bn = n;
        }
        const uint32_t id = d.ids[cur][i];
        const float4 lo = d.plo[id], hi = d.phi[id], c = d.pc[id];
        b[0] = fminf(b[0], lo.x); b[1] = fminf(b[1], lo.y); b[2] = fminf(b[2], lo.z);
        b[3] = fmaxf(b[3], hi.x); b[4] = fmaxf(b[4], hi.y); b[5] = fmaxf(b[5], hi.z);
        b[6] = fminf(b[6], c.x); b[7] = fminf(b[7], c.y); b[8] = fminf(b[8], c.z);
        b[9] = fmaxf(b[9], c.x); b[10] = fmaxf(b[10], c.y); b[11] = fmaxf(b[11], c.z);
    }
    if (one < 0) {
        if (bn >= 0) flush(d.nb + 6 * bn, d.cb + 6 * bn);
        return;
    }
    // one node: warp reduction (lanes without positions hold the empty box), lane 0 to shared
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const float o = __shfl_xor_sync(0xffffffffu, b[k], off);
            b[k] = (k % 6) < 3 ? fminf(b[k], o) : fmaxf(b[k], o);
        }
    }
    if ((threadIdx.x & 31u) == 0) flush(s, s + 6);
    __syncthreads();
    if (threadIdx.x < 3) {
        amin(d.nb + 6 * one + threadIdx.x, s[threadIdx.x]);
        amax(d.nb + 6 * one + 3 + threadIdx.x, s[3 + threadIdx.x]);
        amin(d.cb + 6 * one + threadIdx.x, s[6 + threadIdx.x]);
        amax(d.cb + 6 * one + 3 + threadIdx.x, s[9 + threadIdx.x]);
    }
}

// per-axis bins of the centroids over each active node's centroid bounds
__global__ void __launch_bounds__(256) k_bin(Dev d, int cur, uint32_t nt) {
    __shared__ float sb[3 * kBins * 6];
    __shared__ uint32_t sc[3 * kBins];
    const uint32_t p0 = blockIdx.x * kChunk, p1 = min(nt, p0 + kChunk);
    const int32_t* pn = d.pn[cur];
    const int32_t one = block_node(pn, p0, p1);
    for (uint32_t i = threadIdx.x; i < 3u * kBins * 6u; i += blockDim.x) sb[i] = (i % 6u) < 3 ? kBig : -kBig;
    for (uint32_t i = threadIdx.x; i < 3u * kBins; i += blockDim.x) sc[i] = 0;
    __syncthreads();
    for (uint32_t i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
        const int32_t n = pn[i];
        if (n < 0) continue;
        const uint32_t id = d.ids[cur][i];
        const float4 lo = d.plo[id], hi = d.phi[id], c = d.pc[id];
        const float* cb = d.cb + 6 * n;
        const float cc[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; ++a) {
            const float ext = cb[3 + a] - cb[a];
            if (!(ext > 0.f)) continue;
            const float scale = (float)kBins / ext;
            const int b = bin_of(cc[a], cb[a], scale);
            if (one >= 0) {
                float* bx = sb + (a * kBins + b) * 6;
                amin_s(bx + 0, lo.x); amin_s(bx + 1, lo.y); amin_s(bx + 2, lo.z);
                amax_s(bx + 3, hi.x); amax_s(bx + 4, hi.y); amax_s(bx + 5, hi.z);
                atomicAdd(sc + a * kBins + b, 1u);
            } else {
                float* bx = d.bb + ((size_t)(n * 3 + a) * kBins + b) * 6;
                amin(bx + 0, lo.x); amin(bx + 1, lo.y); amin(bx + 2, lo.z);
                amax(bx + 3, hi.x); amax(bx + 4, hi.y); amax(bx + 5, hi.z);
                atomicAdd(d.bc + (size_t)(n * 3 + a) * kBins + b, 1u);
            }
        }
    }
    if (one < 0) return;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 3u * kBins; i += blockDim.x) {
        if (!sc[i]) continue;
        float* bx = d.bb + ((size_t)one * 3 * kBins + i) * 6;
        amin(bx + 0, sb[i * 6 + 0]); amin(bx + 1, sb[i * 6 + 1]); amin(bx + 2, sb[i * 6 + 2]);
        amax(bx + 3, sb[i * 6 + 3]); amax(bx + 4, sb[i * 6 + 4]); amax(bx + 5, sb[i * 6 + 5]);
        atomicAdd(d.bc + (size_t)one * 3 * kBins + i, sc[i]);
    }
}

// schedule a child: a next-level active node, or a small node; returns its active index or -1
__device__ __forceinline__ int32_t schedule(Dev& d, int nxt, uint32_t first, uint32_t count, uint32_t out,
                                            uint32_t depth) {
    if (count <= kSmall) {
        const uint32_t k = atomicAdd(&d.counters[2], 1u);
        d.small[k] = make_uint4(first, count, out, depth);
        return -1;
    }
    const uint32_t k = atomicAdd(&d.counters[1], 1u);
    d.act[nxt][k] = make_uint4(first, count, out, depth);
    return (int32_t)k;
}

// one warp per active node, lane b holding bin b: the host builder's SAH sweep (more than kSmall
// triangles: no leaf test) and the children's scheduling.  The right-hand and left-hand boxes and
// counts are suffix and prefix scans over the lanes (min / max and integer sums: exact, so equal
// to the host's sequential sweep), each split's cost is the host's expression, and the cheapest
// split is the first in (axis, bin) order, as the host's strict comparison picks it.
__global__ void __launch_bounds__(128) k_split(Dev d, int cur, uint32_t na) {
    const uint32_t n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = (int)(threadIdx.x & 31u);
    if (n >= na) return;                               // whole warps leave together
    const uint4 A = d.act[cur][n];
    const uint32_t first = A.x, count = A.y;
    const float* nb = d.nb + 6 * n;
    const float* cb = d.cb + 6 * n;
    float best = 3.4e38f;
    int bidx = 0x7fffffff;                             // axis * kBins + bin of the best split
    uint32_t lcnt_at[3];
    for (int ax = 0; ax < 3; ++ax) {
        lcnt_at[ax] = 0;
        const float ext = cb[3 + ax] - cb[ax];
        if (!(ext > 0.f)) continue;
        const float* bb = d.bb + ((size_t)(n * 3 + ax) * kBins + lane) * 6;
        const uint32_t c0 = d.bc[(size_t)(n * 3 + ax) * kBins + lane];
        float rlo[3] = {bb[0], bb[1], bb[2]}, rhi[3] = {bb[3], bb[4], bb[5]};
        float llo[3] = {bb[0], bb[1], bb[2]}, lhi[3] = {bb[3], bb[4], bb[5]};
        uint32_t rc = c0, lc = c0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            float t[6];
            uint32_t tc;
            // suffix: bins lane .. 31
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                t[k] = __shfl_down_sync(0xffffffffu, rlo[k], off);
                t[3 + k] = __shfl_down_sync(0xffffffffu, rhi[k], off);
            }
            tc = __shfl_down_sync(0xffffffffu, rc, off);
            if (lane + off < 32) {
#pragma unroll
                for (int k = 0; k < 3; ++k) { rlo[k] = fminf(rlo[k], t[k]); rhi[k] = fmaxf(rhi[k], t[3 + k]); }
                rc += tc;
            }
            // prefix: bins 0 .. lane
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                t[k] = __shfl_up_sync(0xffffffffu, llo[k], off);
                t[3 + k] = __shfl_up_sync(0xffffffffu, lhi[k], off);
            }
            tc = __shfl_up_sync(0xffffffffu, lc, off);
            if (lane >= off) {
#pragma unroll
                for (int k = 0; k < 3; ++k) { llo[k] = fminf(llo[k], t[k]); lhi[k] = fmaxf(lhi[k], t[3 + k]); }
                lc += tc;
            }
        }
        // split after bin `lane`: left = bins 0..lane, right = bins lane+1..31
        const float ra = area(rlo, rhi);
        const float ra_next = __shfl_down_sync(0xffffffffu, ra, 1);
        const uint32_t rc_next = __shfl_down_sync(0xffffffffu, rc, 1);
        lcnt_at[ax] = lc;
        if (lane < kBins - 1 && lc != 0 && rc_next != 0) {
            const float cost = area(llo, lhi) * (float)lc + ra_next * (float)rc_next;
            if (cost < best) { best = cost; bidx = ax * kBins + lane; }
        }
    }
    // first minimum over the lanes in (axis, bin) order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
        if (ob < best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    const int bax = bidx == 0x7fffffff ? -1 : bidx / kBins;
    const int bsplit = bidx == 0x7fffffff ? -1 : bidx % kBins;
    // left count = the prefix count at the split bin (lane bsplit of that axis's scan)
    uint32_t nl_ax = 0;
    for (int ax = 0; ax < 3; ++ax) {
        const uint32_t v = __shfl_sync(0xffffffffu, lcnt_at[ax], bsplit < 0 ? 0 : bsplit);
        if (ax == bax) nl_ax = v;
    }
    if (lane != 0) return;
    const uint32_t nl = bax < 0 ? count / 2 : nl_ax;    // median split by position without a SAH split
    const uint32_t base = atomicAdd(&d.counters[0], 2u);
    BinNode& o = d.nodes[A.z];
    for (int k = 0; k < 3; ++k) { o.lo[k] = nb[k]; o.hi[k] = nb[3 + k]; }
    o.left = (int32_t)base;
    o.right = (int32_t)base + 1;
    o.first = 0;
    o.count = 0;
    o.n_tris = count;
    atomicMax(&d.counters[3], A.w + 1u);
    d.d_ax[n] = bax;
    d.d_split[n] = bsplit;
    d.d_nl[n] = nl;
    d.d_scale[n] = bax >= 0 ? (float)kBins / (cb[3 + bax] - cb[bax]) : 0.f;
    d.d_child[2 * n] = schedule(d, cur ^ 1, first, nl, base, A.w + 1u);
    d.d_child[2 * n + 1] = schedule(d, cur ^ 1, first + nl, count - nl, base + 1, A.w + 1u);
}

// triangles into their child's range (order within a child is arbitrary: min/max and counts do
// not depend on it); finished positions are carried over unchanged.  The lanes of a warp going
// to the same child take their slots with one atomic (iterations are warp-uniform).
__global__ void k_partition(Dev d, int cur, uint32_t nt) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < nt; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        int32_t n = -1, key = -1, side = 0;
        uint32_t id = 0, pos = i, first = 0, nl = 0;
        if (i < nt) {
            n = d.pn[cur][i];
            id = d.ids[cur][i];
            if (n >= 0) {
                first = d.act[cur][n].x;
                nl = d.d_nl[n];
                const int32_t ax = d.d_ax[n];
                if (ax < 0) {
                    side = i - first >= nl ? 1 : 0;
                } else {
                    const float* cb = d.cb + 6 * n;
                    const float4 c = d.pc[id];
                    const float cc = ax == 0 ? c.x : (ax == 1 ? c.y : c.z);
                    side = bin_of(cc, cb[ax], d.d_scale[n]) > d.d_split[n] ? 1 : 0;
                    key = 2 * n + side;
                }
            }
        }
        const unsigned grp = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(grp) - 1;
        uint32_t base = 0;
        if (key >= 0 && (int)lane == leader)
            base = atomicAdd(side ? &d.rcur[n] : &d.lcur[n], (uint32_t)__popc(grp));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (i >= nt) continue;
        if (n < 0) {
            d.ids[cur ^ 1][i] = id;
            d.pn[cur ^ 1][i] = -1;
            continue;
        }
        if (key >= 0) pos = (side ? first + nl : first) + base + (uint32_t)__popc(grp & lt);
        d.ids[cur ^ 1][pos] = id;
        d.pn[cur ^ 1][pos] = d.d_child[2 * n + side];
    }
}

// one thread per small node: the host builder's small-node path to the leaves
__global__ void k_small(Dev d, int cur, uint32_t ns) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    const uint4 S = d.small[k];
    const uint32_t base = S.x, n = S.y;
    float plo[kSmall][3], phi[kSmall][3], pc[kSmall][3];
    uint32_t pid[kSmall];
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t id = d.ids[cur][base + i];
        const float4 lo = d.plo[id], hi = d.phi[id], c = d.pc[id];
        plo[i][0] = lo.x; plo[i][1] = lo.y; plo[i][2] = lo.z;
        phi[i][0] = hi.x; phi[i][1] = hi.y; phi[i][2] = hi.z;
        pc[i][0] = c.x; pc[i][1] = c.y; pc[i][2] = c.z;
        pid[i] = id;
    }
    struct Item { uint32_t first, count, out, depth; };
    Item st[2 * kSmall];
    int sp = 0;
    st[sp++] = {0, n, S.z, S.w};
    uint32_t maxd = 0;
    while (sp > 0) {
        const Item it = st[--sp];
        const uint32_t f = it.first, c = it.count;
        BinNode& o = d.nodes[it.out];
        float nlo[3], nhi[3], clo[3], chi[3];
        box_empty(nlo, nhi);
        box_empty(clo, chi);
        for (uint32_t i = f; i < f + c; ++i) {
            box_grow(nlo, nhi, plo[i], phi[i]);
            box_grow(clo, chi, pc[i], pc[i]);
        }
        for (int q = 0; q < 3; ++q) { o.lo[q] = nlo[q]; o.hi[q] = nhi[q]; }
        maxd = max(maxd, it.depth);
        bool leaf = c <= d.max_leaf && c <= 2u;
        float best = 3.4e38f;
        int bax = -1, bsplit = -1;
        if (!leaf) {
            for (int ax = 0; ax < 3; ++ax) {
                const float ext = chi[ax] - clo[ax];
                if (!(ext > 0.f)) continue;
                const float scale = (float)kBins / ext;
                int bins[kSmall];
                uint32_t occupied = 0;
                for (uint32_t i = 0; i < c; ++i) {
                    bins[i] = bin_of(pc[f + i][ax], clo[ax], scale);
                    occupied |= 1u << bins[i];
                }
                const int top = 31 - __clz(occupied);
                for (uint32_t m = occupied & ~(1u << top); m; m &= m - 1) {
                    const int v = __ffs(m) - 1;
                    float llo[3], lhi[3], rlo[3], rhi[3];
                    box_empty(llo, lhi);
                    box_empty(rlo, rhi);
                    uint32_t nl = 0, nr = 0;
                    for (uint32_t i = 0; i < c; ++i) {
                        if (bins[i] <= v) { box_grow(llo, lhi, plo[f + i], phi[f + i]); ++nl; }
                        else { box_grow(rlo, rhi, plo[f + i], phi[f + i]); ++nr; }
                    }
                    const float cost = area(llo, lhi) * (float)nl + area(rlo, rhi) * (float)nr;
                    if (cost < best) { best = cost; bax = ax; bsplit = v; }
                }
            }
            if (c <= d.max_leaf) {
                const float leaf_cost = area(nlo, nhi) * (float)c;
                if (bax < 0 || best + area(nlo, nhi) >= leaf_cost) leaf = true;
            }
        }
        if (leaf) {
            o.left = -1; o.right = -1;
            o.first = base + f; o.count = c; o.n_tris = c;
            continue;
        }
        uint32_t mid;
        if (bax < 0) {
            mid = f + c / 2;
        } else {
            const float scale = (float)kBins / (chi[bax] - clo[bax]);
            uint32_t i = f, j = f + c;
            while (true) {
                while (i < j && bin_of(pc[i][bax], clo[bax], scale) <= bsplit) ++i;
                while (i < j && bin_of(pc[j - 1][bax], clo[bax], scale) > bsplit) --j;
                if (i >= j) break;
                for (int q = 0; q < 3; ++q) {
                    float t0 = plo[i][q]; plo[i][q] = plo[j - 1][q]; plo[j - 1][q] = t0;
                    float t1 = phi[i][q]; phi[i][q] = phi[j - 1][q]; phi[j - 1][q] = t1;
                    float t2 = pc[i][q]; pc[i][q] = pc[j - 1][q]; pc[j - 1][q] = t2;
                }
                const uint32_t t3 = pid[i]; pid[i] = pid[j - 1]; pid[j - 1] = t3;
            }
            mid = i;
            if (mid == f || mid == f + c) mid = f + c / 2;
        }
        const uint32_t ob = atomicAdd(&d.counters[0], 2u);
        o.left = (int32_t)ob; o.right = (int32_t)ob + 1;
        o.first = 0; o.count = 0; o.n_tris = c;
        st[sp++] = {mid, f + c - mid, ob + 1, it.depth + 1};
        st[sp++] = {f, mid - f, ob, it.depth + 1};
    }
    for (uint32_t i = 0; i < n; ++i) d.ids[cur][base + i] = pid[i];
    atomicMax(&d.counters[3], maxd);
}

// ---- four-child collapse on the device (the rules of finish_bvh in bvh_build.cpp) ----

// each four-child root of this level picks its children: start from the binary children and
// open the interior child of largest area (the first on ties) while fewer than four; interior
// children become the next level's roots
__global__ void k_collapse(const BinNode* __restrict__ nodes, uint32_t* q, uint32_t lo, uint32_t n,
                           uint32_t* next, int4* kids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t nd = q[lo + i];
    int32_t c[4] = {nodes[nd].left, nodes[nd].right, -1, -1};
    int k = 2;
    while (k < 4) {
        int best = -1;
        float ba = -1.0f;
        for (int j = 0; j < k; ++j) {
            const BinNode& b = nodes[c[j]];
            if (b.left < 0) continue;
            const float a = area(b.lo, b.hi);
            if (a > ba) { ba = a; best = j; }
        }
        if (best < 0) break;
        const BinNode& b = nodes[c[best]];
        for (int j = k; j > best + 1; --j) c[j] = c[j - 1];
        c[best] = b.left;
        c[best + 1] = b.right;
        ++k;
    }
    kids[nd] = make_int4(c[0], c[1], c[2], c[3]);
    for (int j = 0; j < 4; ++j)
        if (c[j] >= 0 && nodes[c[j]].left >= 0) q[atomicAdd(next, 1u)] = (uint32_t)c[j];
}

// four-child nodes in each subtree (deepest level first)
__global__ void k_count4(const BinNode* __restrict__ nodes, const uint32_t* q, uint32_t lo, uint32_t n,
                         const int4* kids, uint32_t* n4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t nd = q[lo + i];
    const int4 c4 = kids[nd];
    const int32_t c[4] = {c4.x, c4.y, c4.z, c4.w};
    uint32_t cnt = 1;
    for (int j = 0; j < 4; ++j)
        if (c[j] >= 0 && nodes[c[j]].left >= 0) cnt += n4[c[j]];
    n4[nd] = cnt;
}

// the node at its depth-first preorder index (children in order, leaf triangles in the same
// order; boxes one ulp outward), its children's indices and triangle offsets for the next level
__global__ void k_place4(const BinNode* __restrict__ nodes, const uint32_t* __restrict__ ids, const uint32_t* q,
                         uint32_t lo, uint32_t n, const int4* kids, const uint32_t* n4, uint32_t* gidx, uint32_t* toff,
                         GpuNode* out, uint32_t* order, uint32_t* leaves) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t nd = q[lo + i];
    const int4 c4 = kids[nd];
    const int32_t c[4] = {c4.x, c4.y, c4.z, c4.w};
    GpuNode g;
    uint32_t gnext = gidx[nd] + 1, t = toff[nd];
    for (int j = 0; j < 4; ++j) {
        if (c[j] < 0) {
            g.lox[j] = g.hix[j] = g.loy[j] = g.hiy[j] = g.loz[j] = g.hiz[j] = 0.0f;
            g.child[j] = ~(int32_t)0;           // leaf of 0 triangles: never entered
            continue;
        }
        const BinNode& b = nodes[c[j]];
        float blo[3] = {b.lo[0], b.lo[1], b.lo[2]}, bhi[3] = {b.hi[0], b.hi[1], b.hi[2]};
        for (int k = 0; k < 3; ++k) {
            if (blo[k] <= bhi[k]) {
                blo[k] = nextafterf(blo[k], -INFINITY);
                bhi[k] = nextafterf(bhi[k], INFINITY);
            }
        }
        g.lox[j] = blo[0]; g.hix[j] = bhi[0];
        g.loy[j] = blo[1]; g.hiy[j] = bhi[1];
        g.loz[j] = blo[2]; g.hiz[j] = bhi[2];
        if (b.left >= 0) {
            g.child[j] = (int32_t)gnext;
            gidx[c[j]] = gnext;
            toff[c[j]] = t;
            gnext += n4[c[j]];
        } else {
            for (uint32_t k = 0; k < b.count; ++k) order[t + k] = ids[b.first + k];
            g.child[j] = ~(int32_t)((t << 3) | b.count);
            atomicAdd(leaves, 1u);
        }
        t += b.n_tris;
    }
    g.pad[0] = g.pad[1] = g.pad[2] = g.pad[3] = 0;
    const float4* src = reinterpret_cast<const float4*>(&g);
    float4* dst = reinterpret_cast<float4*>(out + gidx[nd]);
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[k] = src[k];
}

template <class T>
T* pool_alloc(size_t count, cudaStream_t s, std::vector<void*>& held) {
    int dev = 0;
    TR_CUDA(cudaGetDevice(&dev));
    void* p = nullptr;
    TR_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(1, count) * sizeof(T), tri::device_pool(dev), s));
    held.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

// Builds the four-child BVH of device-resident vertices [nv][3] and triangles [nt][3]; returns
// false when the input is invalid (out-of-range index or non-finite vertex: the caller's host
// builder reports which).  Throws tri::CudaError on CUDA failures.
bool build_bvh_device(const float* d_v, uint32_t nv, const uint32_t* d_t, uint32_t nt, uint32_t max_leaf,
                      cudaStream_t s, const std::function<GpuNode*(size_t)>& alloc_nodes, uint32_t* d_order,
                      DeviceBvh& out) {
    const auto t0 = std::chrono::steady_clock::now();
    if (nt == 0 || nt >= (1u << 28)) return false;
    if (max_leaf < 1 || max_leaf > 7) max_leaf = 4;
    std::vector<void*> held;
    struct Free {
        std::vector<void*>& h; cudaStream_t s;
        ~Free() { for (void* p : h) cudaFreeAsync(p, s); cudaStreamSynchronize(s); }
    } release{held, s};
    const uint32_t amax = nt / (kSmall + 1) + 2;      // active nodes of a level (> kSmall triangles each)
    Dev d{};
    d.max_leaf = max_leaf;
    d.plo = pool_alloc<float4>(nt, s, held);
    d.phi = pool_alloc<float4>(nt, s, held);
    d.pc = pool_alloc<float4>(nt, s, held);
    for (int b = 0; b < 2; ++b) {
        d.ids[b] = pool_alloc<uint32_t>(nt, s, held);
        d.pn[b] = pool_alloc<int32_t>(nt, s, held);
        d.act[b] = pool_alloc<uint4>(amax, s, held);
    }
    d.nb = pool_alloc<float>((size_t)amax * 6, s, held);
    d.cb = pool_alloc<float>((size_t)amax * 6, s, held);
    d.bb = pool_alloc<float>((size_t)amax * 3 * kBins * 6, s, held);
    d.bc = pool_alloc<uint32_t>((size_t)amax * 3 * kBins, s, held);
    d.d_ax = pool_alloc<int32_t>(amax, s, held);
    d.d_split = pool_alloc<int32_t>(amax, s, held);
    d.d_nl = pool_alloc<uint32_t>(amax, s, held);
    d.d_scale = pool_alloc<float>(amax, s, held);
    d.d_child = pool_alloc<int32_t>(2 * (size_t)amax, s, held);
    d.lcur = pool_alloc<uint32_t>(amax, s, held);
    d.rcur = pool_alloc<uint32_t>(amax, s, held);
    d.small = pool_alloc<uint4>(nt, s, held);
    d.nodes = pool_alloc<BinNode>(2 * (size_t)nt, s, held);
    d.counters = pool_alloc<uint32_t>(8, s, held);

    const uint32_t grid_nt = std::max(1u, std::min(8192u, (nt + 255) / 256));
    uint32_t h[8] = {1, 0, 0, 0, 0, 0, 0, 0};         // the root is node 0
    TR_CUDA(cudaMemcpyAsync(d.counters, h, sizeof(h), cudaMemcpyHostToDevice, s));
    k_prims<<<grid_nt, 256, 0, s>>>(d_v, nv, d_t, nt, d);
    TR_CUDA(cudaGetLastError());
    // the root: a level node, or directly a small node
    const uint4 root = make_uint4(0, nt, 0, 0);
    uint32_t na = 0, nsmall = 0;
    if (nt > kSmall) {
        TR_CUDA(cudaMemcpyAsync(d.act[0], &root, sizeof(root), cudaMemcpyHostToDevice, s));
        na = 1;
    } else {
        TR_CUDA(cudaMemcpyAsync(d.small, &root, sizeof(root), cudaMemcpyHostToDevice, s));
        nsmall = 1;
        const uint32_t one = 1;
        TR_CUDA(cudaMemcpyAsync(d.counters + 2, &one, sizeof(one), cudaMemcpyHostToDevice, s));
    }
    int cur = 0;
    const uint32_t chunks = (nt + kChunk - 1) / kChunk;
    while (na) {
        k_clear<<<std::max(1u, std::min(4096u, (na * 3u * kBins * 6u + 255) / 256)), 256, 0, s>>>(d, na);
        k_bounds<<<chunks, 256, 0, s>>>(d, cur, nt);
        k_bin<<<chunks, 256, 0, s>>>(d, cur, nt);
        TR_CUDA(cudaMemsetAsync(d.counters + 1, 0, sizeof(uint32_t), s));
        k_split<<<(na + 3) / 4, 128, 0, s>>>(d, cur, na);      // one warp per active node
        k_partition<<<grid_nt, 256, 0, s>>>(d, cur, nt);
        TR_CUDA(cudaGetLastError());
        cur ^= 1;
        TR_CUDA(cudaMemcpyAsync(h, d.counters, sizeof(h), cudaMemcpyDeviceToHost, s));
        TR_CUDA(cudaStreamSynchronize(s));
        if (h[4]) return false;                       // invalid input
        na = h[1];
        nsmall = h[2];
    }
    if (nsmall) {
        k_small<<<(nsmall + 127) / 128, 128, 0, s>>>(d, cur, nsmall);
        TR_CUDA(cudaGetLastError());
    }
    TR_CUDA(cudaMemcpyAsync(h, d.counters, sizeof(h), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    if (h[4]) return false;
    const uint32_t nnodes = h[0];
    BinNode top;
    TR_CUDA(cudaMemcpyAsync(&top, d.nodes, sizeof(top), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    if (top.left < 0) return false;                 // a one-leaf scene: the host builder takes it

    // collapse to four-child nodes, level by level from the root
    uint32_t* q = pool_alloc<uint32_t>(nnodes, s, held);
    int4* kids = pool_alloc<int4>(nnodes, s, held);
    uint32_t* n4 = pool_alloc<uint32_t>(nnodes, s, held);
    uint32_t* gidx = pool_alloc<uint32_t>(nnodes, s, held);
    uint32_t* toff = pool_alloc<uint32_t>(nnodes, s, held);
    const uint32_t zero = 0;
    TR_CUDA(cudaMemcpyAsync(q, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
    TR_CUDA(cudaMemcpyAsync(gidx, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
    TR_CUDA(cudaMemcpyAsync(toff, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> lvl_lo{0}, lvl_n{1};
    while (true) {
        const uint32_t lo = lvl_lo.back(), n = lvl_n.back();
        const uint32_t next0 = lo + n;
        TR_CUDA(cudaMemcpyAsync(d.counters + 5, &next0, sizeof(next0), cudaMemcpyHostToDevice, s));
        k_collapse<<<(n + 127) / 128, 128, 0, s>>>(d.nodes, q, lo, n, d.counters + 5, kids);
        TR_CUDA(cudaGetLastError());
        uint32_t next = 0;
        TR_CUDA(cudaMemcpyAsync(&next, d.counters + 5, sizeof(next), cudaMemcpyDeviceToHost, s));
        TR_CUDA(cudaStreamSynchronize(s));
        if (next == next0) break;
        lvl_lo.push_back(next0);
        lvl_n.push_back(next - next0);
    }
    const int levels = (int)lvl_lo.size();
    for (int L = levels - 1; L >= 0; --L)
        k_count4<<<(lvl_n[L] + 127) / 128, 128, 0, s>>>(d.nodes, q, lvl_lo[L], lvl_n[L], kids, n4);
    uint32_t n4root = 0;
    TR_CUDA(cudaMemcpyAsync(&n4root, n4, sizeof(n4root), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    GpuNode* dn = alloc_nodes(n4root);
    TR_CUDA(cudaMemsetAsync(d.counters + 6, 0, sizeof(uint32_t), s));
    for (int L = 0; L < levels; ++L)
        k_place4<<<(lvl_n[L] + 127) / 128, 128, 0, s>>>(d.nodes, d.ids[cur], q, lvl_lo[L], lvl_n[L], kids, n4,
                                                          gidx, toff, dn, d_order, d.counters + 6);
    TR_CUDA(cudaGetLastError());
    uint32_t leaves = 0;
    TR_CUDA(cudaMemcpyAsync(&leaves, d.counters + 6, sizeof(leaves), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    out.nodes = n4root;
    out.depth = (uint32_t)levels;
    out.stack = 3 * out.depth + 1;
    out.binary_depth = h[3];
    out.leaves = leaves;
    out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

}  // namespace trh
