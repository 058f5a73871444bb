// Batched multi-view path tracing: many views (each its own camera, image
// size, sample count and running-mean image) of one or more scenes, rendered
// as a few large wavefronts whose whole launch sequence is captured once as
// a CUDA graph and replayed per call.  Each view gets exactly what `spp`
// PBRenderer::render() calls would give it (PBRenderer.cu:137-230,
// PathTracer.cu:97-169 with the running mean of :162-168).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "pathtracer.hpp"

namespace cupbr_b200 {

struct BatchView {   // device table entry
    f3 cam_pos, cam_x, cam_y, cam_z;
    uint32_t width, height, frame0, spp;
    float* img;      // width * height RGB running mean
};

// Frames [first, first + frames) (relative to the view's frame0) of one
// view, as a contiguous run of a wavefront's paths starting at path0; its
// pixels start at pix0 of the wavefront's accumulation grid.
struct BatchSegment {
    uint32_t path0, pix0, view, first, frames;
};

struct BatchWave {
    uint32_t scene;        // index into the batch's scene list
    uint32_t seg0, nseg;   // slice of the segment table
    uint32_t n_paths, n_pixels;
};

// Splits every scene's views into wavefronts of at most `capacity` paths
// (whole frames; a view's frames stay in order).
void batch_plan(const std::vector<uint32_t>& view_scene, const std::vector<BatchView>& views, uint32_t n_scenes,
                uint32_t capacity, std::vector<BatchWave>& waves, std::vector<BatchSegment>& segs);

// Issues one wavefront (counters, camera rays, per depth closest hit / shade /
// shadow rays, accumulation) on `st`; `dsegs` / `dviews` are device tables.
cudaError_t batch_record_wave(const DeviceScene& S, const BatchWave& w, const BatchSegment* dsegs,
                              const BatchView* dviews, const Workspace& W, uint32_t max_depth, int num_sms,
                              cudaStream_t st);

}  // namespace cupbr_b200
