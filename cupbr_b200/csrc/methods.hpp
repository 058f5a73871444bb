// Host interface of the VOLUME, GRADIENTDOMAIN and RAYTRACER kernels (methods.cu).
#pragma once

#include <cuda_runtime.h>

#include "pathtracer.hpp"

namespace cupbr_b200 {

// PBRendering::volumetracing (one frame folded into the running mean) as a
// wavefront over the path tracer's workspace (W sized for F.n_paths paths).
// img == nullptr: the frames' radiance stays in W.radiance (folded later by
// pt_launch_accumulate).
// count_stats: traversal counters into W.stats, ray counts in W.ctr
// (CTR_RAYS: closest-hit rays, CTR_SHADOW: shadow rays, per depth).
cudaError_t volume_render_frame(const DeviceScene& S, const PTFrame& F, const Workspace& W, float* img, cudaStream_t st,
                                int num_sms, bool count_stats);
// F.frames consecutive PBRendering::gradientdomain frames in two steps.
// gdpt_trace_frames: their paths as two wavefronts over the path tracer's
// workspace (W sized for 5 F.frames (w - 2) (h - 2) paths; valid_scratch
// holds 8 B per interior pixel and frame); count_stats: traversal counters
// and ray counts into W.stats.  gdpt_fold_frames: per frame, in order, its
// running means from W's path radiances and the reconstruction of them;
// bufs = {gradient_x, gradient_y, base, gx_forward, gx_backward, gy_forward,
// gy_backward, temp}, `out` receives the reconstruction.
cudaError_t gdpt_trace_frames(const DeviceScene& S, const PTFrame& F, const Workspace& W, void* valid_scratch,
                              cudaStream_t st, int num_sms, bool count_stats);
cudaError_t gdpt_fold_frames(const PTFrame& F, const Workspace& W, float* const bufs[8], float* out, cudaStream_t st);
// The reconstruction half of PBRendering::gradientdomain (init_kernel and
// 50 optimization_kernel passes, GradientDomain.cu:382-401) on given buffers.
cudaError_t launch_gdpt_reconstruct(uint32_t w, uint32_t h, const float* base, const float* gxf, const float* gxb,
                                    const float* gyf, const float* gyb, float* gx, float* gy, float* temp, float* out,
                                    cudaStream_t st);
// PBRendering::raytracing
cudaError_t launch_raytrace(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st);

}  // namespace cupbr_b200
