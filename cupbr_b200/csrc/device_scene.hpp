// Committed (GPU-resident) scene: SAH BVH, primitive tables, objects,
// materials, lights and environment uploaded once, like the device copies
// SceneLoader.cpp:370-453 makes, but as a handful of flat arrays instead of
// one cudaMalloc per object and per BVH node.
#pragma once

#include <string>
#include <vector>

#include "bvh_build.hpp"
#include "dev_common.cuh"
#include "host_scene.hpp"

namespace cupbr_b200 {

struct GpuScene {
    HostScene host;
    bool committed = false;
    BvhBuildParams params;           // BVH parameters of the last commit
    uint64_t generation = 0;         // incremented by every commit (device buffers replaced)
    DeviceScene dev{};
    std::vector<void*> buffers;
    FlatBvh bvh;
    uint64_t device_bytes = 0;
    std::vector<uint32_t> key_base;  // per object: first primitive key
    std::vector<int32_t> key_obj;    // per primitive key: object id
    std::vector<uint32_t> dfs_order; // the reference's object-BVH leaf order
    bool bvh_device = false;         // last commit built the BVH on the GPU
    double bvh_ms = 0.0, commit_ms = 0.0;  // wall times of the last commit

    ~GpuScene();
    void release();
};

// Leaf order of the reference's object BVH (BoundingVolumeHierarchy.cpp:46-136).
std::vector<uint32_t> reference_object_order(const HostScene& sc);

bool commit_scene(GpuScene& g, const BvhBuildParams& p, std::string& err);

// Device record of a material (materials are stored one per object).
DMaterial device_material(const HMaterial& m);

}  // namespace cupbr_b200
