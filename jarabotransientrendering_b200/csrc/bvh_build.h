// bvh_build.h - host-side BVH construction for the GPU traversal kernels.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace trh {

// 128-byte four-child node, read by the kernels as eight 16-byte vector loads:
//   q0..q5 = child bounds lo.x[4], hi.x[4], lo.y[4], hi.y[4], lo.z[4], hi.z[4]
//   q6 = child refs[4], q7 = padding
// ref >= 0: interior node index; ref < 0: leaf, ~ref = (first_triangle << 3) | count
// (count 0: empty slot, never entered).
struct alignas(16) GpuNode {
    float lox[4], hix[4], loy[4], hiy[4], loz[4], hiz[4];
    int32_t child[4];
    int32_t pad[4];
};
static_assert(sizeof(GpuNode) == 128, "node must be 128 bytes");

// 48-byte triangle in leaf order: v0.xyz + triangle id (bits), v1.xyz, v2.xyz.
struct alignas(16) GpuTri {
    float v0[3]; uint32_t id;
    float v1[3]; float pad1;
    float v2[3]; float pad2;
};
static_assert(sizeof(GpuTri) == 48, "triangle must be 48 bytes");

// Binary SAH tree node (output of the binned builders, input of the four-child collapse).
struct BinNode {
    float lo[3], hi[3];          // bounds of the node's triangles
    int32_t left, right;         // children; left < 0: leaf
    uint32_t first, count;       // leaf: its triangles, [first, first + count) of the id order
    uint32_t n_tris;             // triangles in the subtree
};

struct BvhBuildResult {
    std::vector<GpuNode> nodes;
    std::vector<uint32_t> order;  // triangle ids in leaf order (leaf refs index this order)
    std::vector<GpuTri> tris;     // the triangles in that order (only when write_tris)
    uint32_t depth = 0;          // four-child levels on the deepest path (root = 1)
    uint32_t stack = 0;          // traversal stack entries a ray can need: 3 per level
    uint32_t binary_depth = 0;   // depth of the binary SAH tree it was collapsed from
    uint32_t leaves = 0;
    double build_ms = 0.0;
};

// Binned SAH (32 bins over centroid bounds), leaves of at most `max_leaf` (<= 7) triangles,
// collapsed to four-child nodes (each node opens its largest-area interior children).
// vertices [nv][3], triangles [nt][3].  Returns false (with msg) on bad input.
// write_tris = false leaves `tris` empty: the caller gathers the triangle records from `order`
// (the CUDA path does it on the device).
bool build_bvh(const float* vertices, uint32_t nv, const uint32_t* triangles, uint32_t nt,
               uint32_t max_leaf, BvhBuildResult& out, std::string* msg, bool write_tris = true);

// Collapses a binary tree (root at index 0 of nodes[0, cap), leaves indexing `ids`, the triangle
// ids in leaf order) to four-child nodes and fills out (nodes, order, stack, depths; tris when
// write_tris).  Shared by the host builder and the device builder.
bool finish_bvh(const BinNode* nodes, size_t cap, const uint32_t* ids, uint32_t nt, uint32_t binary_depth,
                const float* vertices, const uint32_t* triangles, bool write_tris, BvhBuildResult& out);

}  // namespace trh
