// Host interface of the post-processing kernels (post.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cupbr_b200 {

// ToneMapper::toneMap: hdr (npix * 3 floats) -> rgba (npix * 4 bytes).
// type 0 = REINHARD (uses exposure), 1 = GAMMA.
cudaError_t launch_tonemap(const float* hdr, uint32_t npix, int type, float exposure, uint8_t* rgba, cudaStream_t st);

// PostProcessor::bloom (pyramid depth 6 semantics).  scratch_half holds
// (w/2) * (h/2) * 3 floats.  With rgba == nullptr the HDR result goes to
// `out`; otherwise the result is tone-mapped into rgba and `out` is unused.
// Requires w >= 2 and h >= 2.
cudaError_t launch_bloom(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* scratch_half, float* out,
                         uint8_t* rgba, int type, float exposure, cudaStream_t st);

}  // namespace cupbr_b200
