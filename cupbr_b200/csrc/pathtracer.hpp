// Host interface of the wavefront path tracer and its device workspace.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_common.cuh"

namespace cupbr_b200 {

constexpr int PT_TRACE_THREADS = 128;
constexpr uint32_t PT_MAX_DEPTH = 64;

// counter block (one cudaMemsetAsync per frame)
constexpr uint32_t CTR_RAYS = 0;      // [d]: entries in ray queue d
constexpr uint32_t CTR_EFETCH = 64;   // [d]: work-fetch cursor of k_extend(d)
constexpr uint32_t CTR_SHADOW = 128;  // [d]: entries in the shadow queue at depth d
constexpr uint32_t CTR_CFETCH = 192;  // [d]: work-fetch cursor of k_connect(d)
constexpr uint32_t CTR_TFETCH = 256;  // [d]: work-fetch cursor of the medium's transmittance kernel
constexpr uint32_t CTR_FFETCH = 320;  // [d]: work-fetch cursor of the medium's free-flight kernel
constexpr uint32_t CTR_MVERT = 384;   // [d]: medium vertices of depth d
constexpr uint32_t CTR_SVERT = 448;   // [d]: surface vertices of depth d
constexpr uint32_t CTR_TOTAL = 512;

constexpr uint32_t ERR_STACK = 0;     // traversal stack overflows (entries dropped)
constexpr uint32_t ERR_TOTAL = 8;

constexpr uint32_t STAT_EXT_NODES = 0, STAT_EXT_TRIS = 1, STAT_SH_NODES = 2, STAT_SH_TRIS = 3;
// closest-hit and occlusion rays (counted on the device by the per-pixel
// methods; the path tracer counts its rays from the queue counters)
constexpr uint32_t STAT_EXT_RAYS = 4, STAT_SH_RAYS = 5, STAT_TOTAL = 6;

// One wavefront: `frames` consecutive sample frames of one view
// (n_paths = frames * width * height, path p = frame (p / pixels), pixel
// (p % pixels)); frame_index is the first frame's index.
struct PTFrame {
    uint32_t width, height, n_paths, frame_index, max_depth, use_rr;
    uint32_t pixels, frames;
    f3 cam_pos, cam_x, cam_y, cam_z;  // Camera.h:71-74
    uint32_t estimator = 0;           // CUPBR_ESTIMATOR_REFERENCE (0) or CUPBR_ESTIMATOR_PHYSICAL (1)
};

// Device buffers of one renderer (sized for width * height paths).
struct Workspace {
    float4* radiance;      // per path
    float4* rays[2];       // ping-pong ray queues, 3 float4 per slot: (o, path), (d, seed), (throughput, 0)
    float2* hits;          // per ray-queue slot: (t, primitive ref)
    float4* shadow;        // 3 float4 per slot: (origin, light distance), (dir, path), (contribution, 0)
    uint32_t* ctr;         // CTR_TOTAL counters
    uint32_t* err;         // ERR_TOTAL error counters (never reset by a frame)
    uint64_t* stats;       // STAT_TOTAL traversal counters (instrumented frames only)
    uint32_t smem_nodes;   // BVH nodes staged in shared memory per block
    int trace_blocks_per_sm;
};

int pt_occupancy_blocks(int smem_bytes);
// The path tracer's persistent traversal stages on their own: closest hits of
// ray queue[depth] into W.hits, and the shadow queue of depth (3 float4 per
// entry: (origin, distance), (direction, path), (contribution, -)) with the
// visible contributions added to W.radiance[path].
// min_count: the kernel does nothing when the queue holds fewer rays (a
// cached frame's tail kernel takes them).
// count: traversal counters into W.stats (instrumented frames).
cudaError_t pt_launch_extend(const DeviceScene& S, const Workspace& W, uint32_t depth, int num_sms, cudaStream_t st,
                             uint32_t min_count = 0, bool count = false);
// Closest hits of the camera-ray queue (depth 0, filled by k_camera in 8x4
// pixel tiles) traversed as warp packets; same hits as pt_launch_extend.
cudaError_t pt_launch_extend_camera(const DeviceScene& S, const Workspace& W, int num_sms, cudaStream_t st,
                                    uint32_t min_count = 0);
cudaError_t pt_launch_connect(const DeviceScene& S, const Workspace& W, uint32_t depth, int num_sms, cudaStream_t st,
                              bool count = false);
// The path tracer's shading stage of ray queue[depth] (reads F.max_depth and
// F.use_rr only).
cudaError_t pt_launch_shade(const DeviceScene& S, const PTFrame& F, const Workspace& W, uint32_t depth, int num_sms,
                            cudaStream_t st);
// k_camera (camera rays of every path of F, radiance cleared) and
// k_accumulate (running mean of F's frames into img) on their own.
cudaError_t pt_launch_camera(const PTFrame& F, const Workspace& W, cudaStream_t st);
cudaError_t pt_launch_accumulate(const PTFrame& F, const Workspace& W, float* img, cudaStream_t st);
// closest hit (dist == nullptr: t, primitive ref, key) or visibility (vis)
cudaError_t launch_trace_rays(const DeviceScene& S, uint32_t n, const float* o, const float* d, const float* dist,
                              float* t_out, int32_t* prim_out, uint32_t* key_out, int32_t* vis_out, uint32_t* err,
                              cudaStream_t st);
// ev (optional): 3 + 3 * max_depth events recorded around every stage:
// [0] start, [1] after k_camera, per depth after k_extend / k_shade /
// k_connect, [last] after k_accumulate.
// img == nullptr: the frame is traced but not accumulated (pt_launch_accumulate
// does that, possibly on another stream).
// tail_paths > 0: once a depth's ray queue holds fewer rays, one thread per
// ray traces the rest of its path in one launch (same results; counted in
// the closest-hit stage's events; never on count_stats frames).
cudaError_t pt_render_frame(const DeviceScene& S, const PTFrame& F, const Workspace& W, float* img, cudaStream_t st,
                            int num_sms, bool count_stats, cudaEvent_t* ev = nullptr, uint32_t tail_paths = 0);
inline uint32_t pt_event_count(uint32_t max_depth) { return 3 + 3 * max_depth; }

}  // namespace cupbr_b200
