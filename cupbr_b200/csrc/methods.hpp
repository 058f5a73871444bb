// Host interface of the VOLUME, GRADIENTDOMAIN and RAYTRACER kernels (methods.cu).
#pragma once

#include <cuda_runtime.h>

#include "pathtracer.hpp"

namespace cupbr_b200 {

// PBRendering::volumetracing: one frame folded into the running mean.
// stats (instrumented frames, else null): STAT_* traversal counters added to.
cudaError_t launch_volume(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st,
                          uint64_t* stats = nullptr);
// PBRendering::gradientdomain: bufs = {gradient_x, gradient_y, base, gx_forward,
// gx_backward, gy_forward, gy_backward, temp}; `out` receives the reconstruction.
cudaError_t launch_gdpt(const DeviceScene& S, const PTFrame& F, float* const bufs[8], float* out, uint32_t* err,
                        cudaStream_t st, uint64_t* stats = nullptr);
// The reconstruction half of PBRendering::gradientdomain (init_kernel and
// 50 optimization_kernel passes, GradientDomain.cu:382-401) on given buffers.
cudaError_t launch_gdpt_reconstruct(uint32_t w, uint32_t h, const float* base, const float* gxf, const float* gxb,
                                    const float* gyf, const float* gyb, float* gx, float* gy, float* temp, float* out,
                                    cudaStream_t st);
// PBRendering::raytracing
cudaError_t launch_raytrace(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st);

}  // namespace cupbr_b200
