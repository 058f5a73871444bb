// Heterogeneous medium (density grid): wavefront forward renderer and its
// path-replay adjoint.  No counterpart in the reference: its
// VolumeRenderer.cu renders a homogeneous medium only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "pathtracer.hpp"

namespace cupbr_b200 {

// Free-flight steps per segment before a path is abandoned (and counted as
// an error).  With the majorant times the box diagonal in the tens, a path
// that reaches this is broken input (NaN densities, a zero majorant).
constexpr int MEDIUM_MAX_EVENTS = 1 << 16;
// Parameter gradients are accumulated per block in shared memory up to this
// many entries (32 KB next to the 16 KB of staged BVH nodes), in global
// memory beyond.
constexpr uint32_t MEDIUM_SMEM_PARAMS = 8192;
constexpr uint32_t MEDIUM_STATS = 5;

struct MediumGrid {
    const float* __restrict__ density;  // nz * ny * nx, x fastest
    uint32_t nx, ny, nz;
    f3 lo, hi;       // grid box (world space)
    f3 inv_cell;     // (nx, ny, nz) / (hi - lo)
    float majorant;  // >= every density
    float inv_majorant;  // 1 / majorant
};

struct MediumParams {
    uint32_t width, height, spp, frame0, max_depth;
    float albedo;  // sigma_s / sigma_t of the medium
    float g;       // Henyey-Greenstein asymmetry
    float q;       // 0: analog delta tracking; (0, 1): weighted tracking with real-event probability q
    float inv_q, inv_one_minus_q;  // 1 / q and 1 / (1 - q) (weighted tracking)
    f3 cam_pos, cam_x, cam_y, cam_z;
};

// Device buffers: the path tracer's queues and per-path radiance, plus one
// float4 per shadow-queue slot for the adjoint (RNG state of the ratio
// tracking, light, Lambert object + 1).
struct MediumWorkspace {
    Workspace pt;
    float4* shadow_aux;
    float4* verts;                    // 3 per path: a depth's medium vertices from the front, surface vertices from the back
    uint32_t capacity;                // paths per wavefront
    double* lsum;                     // 3 per path: radiance sums of the gradient's replays
    // Instrumented forward passes (nullptr otherwise) add up: [0] free-flight
    // density lookups, [1] ratio-tracking density lookups, [2] ray-queue
    // entries shaded, [3] shadow rays, [4] paths.
    unsigned long long* stats;
};

// Parameter gradient layout (g_params): [0] medium albedo, then per object
// 3 floats (diffuse albedo, Lambert objects only), then per object 3 floats
// (emission albedo_e), then per light 3 floats (radiance of an area light,
// intensity of a point light).
__host__ __device__ inline uint32_t medium_param_count(uint32_t n_objects, uint32_t n_lights) { return 1 + 6 * n_objects + 3 * n_lights; }
__host__ __device__ inline uint32_t medium_emission_offset(uint32_t n_objects) { return 1 + 3 * n_objects; }
__host__ __device__ inline uint32_t medium_light_offset(uint32_t n_objects) { return 1 + 6 * n_objects; }

inline uint32_t medium_event_count(uint32_t max_depth) { return 3 + 4 * max_depth; }
// Wavefronts medium_render runs: up to W.capacity paths (whole frames) each.
uint32_t medium_batches(const MediumParams& P, const MediumWorkspace& W);
// img (width * height RGB floats) = mean over samples frame0 .. frame0 +
// spp - 1.  ev (optional): medium_event_count(max_depth) events per
// wavefront: [0] start, [1] after the camera kernel, per depth after closest
// hit / shade / transmittance / shadow rays, [last] after the accumulation.
cudaError_t medium_render(const DeviceScene& S, const MediumGrid& G, const MediumParams& P, const MediumWorkspace& W,
                          float* img, uint32_t* err, int num_sms, cudaStream_t st, cudaEvent_t* ev = nullptr);
// Adds dLoss/dtheta to g_grid (nz*ny*nx) and g_params for grad_img =
// dLoss/dimg (width * height RGB).  Requires 0 < q < 1.
cudaError_t medium_gradient(const DeviceScene& S, const MediumGrid& G, const MediumParams& P, const MediumWorkspace& W,
                            const float* grad_img, float* g_grid, float* g_params, uint32_t* err, int num_sms,
                            cudaStream_t st);

}  // namespace cupbr_b200
