// Device (GPU) build of the binned-SAH BVH: the same tree, leaf order and
// flat 4-wide node array as the host builder (bvh_build.cpp), built on the
// GPU.  Large nodes are split level by level with all of their primitives
// binned at once across the GPU; subtrees of at most 960 primitives are
// built one CTA each in shared memory (below 32 primitives, one warp per
// subtree); the 4-wide collapse and the node
// layout (breadth-first top levels, depth-first below) run level by level
// too.  Every split follows the host builder's rules on the same float
// arithmetic, and those rules depend only on which primitives a node holds,
// so the arrays are identical (the SAH cost statistic is a double sum taken
// in another order and can differ in its last bits).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "bvh_build.hpp"

namespace cupbr_b200 {

// boxes[t]: primitive boxes of type t (as for build_bvh); perm[t] receives
// the leaf order; *d_nodes receives a cudaMalloc'd array of *n_nodes 4-wide
// nodes (the caller frees it); out.stats as build_bvh sets them, out.nodes
// a host copy of the root node only.  Work is ordered on `st`; the call
// returns after it has finished.
bool build_bvh_device(const std::vector<PrimBox>* boxes, int ntypes, const uint32_t* slot_offset,
                      const BvhBuildParams& p, std::vector<uint32_t>* perm, FlatBvh& out, float4** d_nodes,
                      uint32_t* n_nodes, cudaStream_t st, std::string& err);

}  // namespace cupbr_b200
