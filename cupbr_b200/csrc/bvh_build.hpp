// Binned-SAH BVH builder (host, OpenMP) and the flat 2-wide node format the
// traversal kernels read.  This replaces the reference's object-level median
// split (BoundingVolumeHierarchy.cpp:46-136) with a primitive-level SAH tree.
//
// GPU node = 64 bytes = 4 x float4 (one 128-bit load each):
//   n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   n3 = (child0, child1, -, -) as int bits
// child >= 0: index of an inner node; child < 0: leaf ~(start << 3 | count-1)
// over the unified primitive slot space (triangles, then spheres, then
// quads); BVH_EMPTY marks a missing child (its box is inverted).
#pragma once

#include <cstdint>
#include <vector>

namespace cupbr_b200 {

constexpr int32_t BVH_EMPTY = (int32_t)0x80000000;
constexpr uint32_t BVH_NODE_F4 = 4;  // float4s per node
constexpr int BVH_MAX_LEAF = 8;

struct PrimBox {
    float lo[3], hi[3];
};

struct BvhBuildParams {
    int max_leaf = 4;         // primitives per leaf (<= BVH_MAX_LEAF)
    float trav_cost = 1.0f;   // SAH cost of one node step relative to one primitive test
    int top_bfs_levels = 10;  // levels laid out breadth-first at the front (shared-memory staging)
};

struct BvhStats {
    uint32_t inner_nodes = 0, leaves = 0, max_depth = 0;
    double sah_cost = 0.0;
};

// A built tree for one primitive type: leaves index perm[] (primitive ids).
struct TypeTree;

struct FlatBvh {
    std::vector<float> nodes;  // 16 floats per node
    BvhStats stats;
};

// Builds one SAH tree per primitive type and joins them under a common root.
// boxes[t] are the primitive boxes of type t; perm[t] receives the leaf order
// (slot s of type t holds primitive perm[t][s]); slot_offset[t] is the first
// unified slot of type t.
void build_bvh(const std::vector<PrimBox>* boxes, int ntypes, const uint32_t* slot_offset, const BvhBuildParams& p,
               std::vector<uint32_t>* perm, FlatBvh& out);

}  // namespace cupbr_b200
