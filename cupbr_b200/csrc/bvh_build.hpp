// Binned-SAH BVH builder (host, std::thread) and the flat 4-wide node format
// the traversal kernels read.  This replaces the reference's object-level
// median split (BoundingVolumeHierarchy.cpp:46-136) with a primitive-level
// SAH tree, built binary and collapsed to 4 children per node.
//
// GPU node = 128 bytes = 8 x float4 (one cache line; 7 are read):
//   n0 = lo.x of children 0..3, n1 = hi.x, n2 = lo.y, n3 = hi.y,
//   n4 = lo.z, n5 = hi.z, n6 = child references 0..3 (int bits), n7 = 0
// child >= 0: index of an inner node; child < 0: leaf ~(start << 3 | count-1)
// over the unified primitive slot space (triangles, then spheres, then
// quads); BVH_EMPTY marks a missing child (its box is inverted).
#pragma once

#include <cstdint>
#include <vector>

namespace cupbr_b200 {

constexpr int32_t BVH_EMPTY = (int32_t)0x80000000;
constexpr uint32_t BVH_NODE_F4 = 8;  // float4s per node
constexpr uint32_t BVH_NODE_BYTES = 16 * BVH_NODE_F4;
constexpr int BVH_MAX_LEAF = 8;

struct PrimBox {
    float lo[3], hi[3];
};

struct BvhBuildParams {
    int max_leaf = 4;         // primitives per leaf (<= BVH_MAX_LEAF)
    float trav_cost = 2.0f;   // SAH cost of one node step relative to one primitive test
    int top_bfs_levels = 4;   // 4-wide levels laid out breadth-first at the front (shared-memory staging)
    bool device = true;       // build on the GPU (bvh_gpu.cu); false: build_bvh on the host (same arrays)
};

struct BvhStats {
    uint32_t inner_nodes = 0, leaves = 0, max_depth = 0;
    double sah_cost = 0.0;
};

// A built tree for one primitive type: leaves index perm[] (primitive ids).
struct TypeTree;

struct FlatBvh {
    std::vector<float> nodes;  // 4 * BVH_NODE_F4 floats per node
    BvhStats stats;
};

// Builds one SAH tree per primitive type and joins them under a common root.
// boxes[t] are the primitive boxes of type t; perm[t] receives the leaf order
// (slot s of type t holds primitive perm[t][s]); slot_offset[t] is the first
// unified slot of type t.
void build_bvh(const std::vector<PrimBox>* boxes, int ntypes, const uint32_t* slot_offset, const BvhBuildParams& p,
               std::vector<uint32_t>* perm, FlatBvh& out);

}  // namespace cupbr_b200
