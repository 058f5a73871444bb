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
    uint32_t scene;  // index into the batch's scene list
};

// Work item of the persistent batch kernel: 32 consecutive queue slots of
// one view (one 8x4 pixel tile, slot_pixel order) through all of the view's
// frames, traced by one warp.
struct BatchItem {
    uint32_t view, slot0;
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

// Grid barrier state of the cooperative batch kernel (zeroed before each launch).
struct BatchBarrier {
    uint32_t count, gen, abort;
};

// Every wavefront of `waves` (batch_plan) in one cooperative launch of
// blocks_per_sm x SMs blocks of 256 threads (0: as many as fit, which the
// cooperative launch requires to be resident together): per wavefront the
// camera, closest-hit, shading, shadow-ray and accumulation stages of the
// wavefront mode, separated by grid barriers whose waits are bounded (a
// barrier that times out sets gb->abort and every block returns).  W is the
// wavefront workspace (sized for the largest wavefront); `scenes` holds the
// batch's DeviceScene records.
// probe_ns > 0 (test hook): block 0 leaves before the first barrier, which
// the others wait on for probe_ns and then abort (no fault, no hang).
cudaError_t batch_launch_coop(const DeviceScene* scenes, const BatchWave* waves, uint32_t n_waves,
                              const BatchSegment* segs, const BatchView* views, const Workspace& W,
                              uint32_t max_depth, uint32_t blocks_per_sm, int num_sms, BatchBarrier* gb,
                              cudaStream_t st, uint64_t probe_ns = 0);
// Resident 256-thread blocks per SM of the cooperative kernel.
int batch_coop_occupancy();

// Work items of every view, heaviest first (frames x the scene's BVH nodes,
// then view and tile order), so the last items to finish are short ones.
void batch_items(const std::vector<BatchView>& views, const std::vector<uint32_t>& scene_nodes,
                 std::vector<BatchItem>& items);

// The persistent batch kernel: THREADS per block (64, 128 or 256),
// blocks_per_sm x SMs blocks; each warp takes items from *counter (zeroed
// first, in the same stream) until n_items are taken and traces its 32
// paths per frame one thread per path (the path tracer's shading and
// traversal), folding the frames into the view's running mean in frame
// order, so every view gets exactly what spp render() calls give it.
// `scenes` is a device array of the batch's DeviceScene records.
// packet: the camera rays of each frame of an item find their hits as one
// warp packet (same hits).
cudaError_t batch_launch_persistent(const DeviceScene* scenes, const BatchView* views, const BatchItem* items,
                                    uint32_t n_items, uint32_t* counter, uint32_t max_depth, uint32_t threads,
                                    uint32_t blocks_per_sm, bool packet, int num_sms, uint32_t* err, cudaStream_t st);
// Resident blocks per SM of the persistent kernel at `threads` per block.
int batch_persistent_occupancy(uint32_t threads, bool packet);

// Deepest path the albedo-texture adjoint records (vertices per path).
constexpr uint32_t BATCH_BWD_MAX_DEPTH = 16;
// Adjoint of the persistent kernel's frames with respect to the scenes'
// albedo textures: grad_tex[scene] (tex_w * tex_h RGB floats, or null) +=
// the derivative of sum over views and pixels of grad_img[view][pixel] .
// image[pixel] (grad_img[view] width * height RGB floats, or null), each
// view's image taken as the mean of its frames 0 .. frame0 + spp - 1 and
// only the frames frame0 .. frame0 + spp - 1 replayed (exact when frame0 = 0).
// max_depth <= BATCH_BWD_MAX_DEPTH.  Same work items and counter protocol
// as the forward kernel.
cudaError_t batch_launch_backward(const DeviceScene* scenes, const BatchView* views, const BatchItem* items,
                                  uint32_t n_items, uint32_t* counter, uint32_t max_depth, const float* const* grad_img,
                                  float* const* grad_tex, uint32_t threads, uint32_t blocks_per_sm, int num_sms,
                                  uint32_t* err, cudaStream_t st);
int batch_backward_occupancy(uint32_t threads);

}  // namespace cupbr_b200
