// bvh_build.h - host-side BVH construction for the GPU traversal kernels.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace trh {

// 64-byte two-child node, read by the kernels as four 16-byte vector loads:
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)   d = (ref0, ref1, 0, 0)
// ref >= 0: interior node index; ref < 0: leaf, ~ref = (first_triangle << 3) | count.
struct alignas(16) GpuNode {
    float a[4], b[4], c[4];
    int32_t d[4];
};
static_assert(sizeof(GpuNode) == 64, "node must be 64 bytes");

// 48-byte triangle in leaf order: v0.xyz + triangle id (bits), v1.xyz, v2.xyz.
struct alignas(16) GpuTri {
    float v0[3]; uint32_t id;
    float v1[3]; float pad1;
    float v2[3]; float pad2;
};
static_assert(sizeof(GpuTri) == 48, "triangle must be 48 bytes");

struct BvhBuildResult {
    std::vector<GpuNode> nodes;
    std::vector<GpuTri> tris;
    uint32_t depth = 0;
    uint32_t leaves = 0;
    double build_ms = 0.0;
};

// Binned SAH (32 bins over centroid bounds), leaves of at most `max_leaf` (<= 7) triangles.
// vertices [nv][3], triangles [nt][3].  Returns false (with msg) on bad input.
bool build_bvh(const float* vertices, uint32_t nv, const uint32_t* triangles, uint32_t nt,
               uint32_t max_leaf, BvhBuildResult& out, std::string* msg);

}  // namespace trh
