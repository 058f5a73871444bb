// Host interface of the post-processing kernels (post.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cupbr_b200 {

// ToneMapper::toneMap: hdr (npix * 3 floats) -> rgba (npix * 4 bytes).
// type 0 = REINHARD (uses exposure), 1 = GAMMA.
cudaError_t launch_tonemap(const float* hdr, uint32_t npix, int type, float exposure, uint8_t* rgba, cudaStream_t st);

// The tone map reads each channel's 8-bit level from per-device tables
// built from the tone-map formulas (identical levels; post.cu).  The first
// tone-mapping call on a device enqueues their build (about a millisecond)
// on its stream; until that has run, kernels evaluate the formulas.
cudaError_t ensure_tone_levels(cudaStream_t st);
// Validation: mismatches[t] = number of 32-bit inputs whose looked-up level
// differs from the formula's (0 expected), flagged[t] = buckets left to the
// formulas, for tables t = REINHARD red/green, REINHARD blue, GAMMA.
// Synchronizes the stream.
cudaError_t verify_tone_levels(unsigned long long mismatches[3], uint32_t flagged[3], cudaStream_t st);

// PostProcessor::bloom (pyramid depth 6 semantics).  scratch_half holds
// (w/2) * (h/2) * 3 floats.  With rgba == nullptr the HDR result goes to
// `out`; otherwise the result is tone-mapped into rgba and `out` is unused.
// Requires w >= 2 and h >= 2.
cudaError_t launch_bloom(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* scratch_half, float* out,
                         uint8_t* rgba, int type, float exposure, cudaStream_t st);

// Bloom with its level-1 scratch in a fixed device array owned by the
// library (no allocation).  At most BLOOM_NOALLOC_MAX_HALF_PIXELS level-1
// pixels, i.e. (w/2) * (h/2) <= 1048576 (inputs up to 2048 x 2048); the
// caller checks the size.  Calls whose work overlaps on the GPU share the
// array and race.
constexpr uint32_t BLOOM_NOALLOC_MAX_HALF_PIXELS = 1024u * 1024u;
constexpr int BLOOM_NOALLOC_MAX_DEVICES = 64;
cudaError_t bloom_static_scratch(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* out,
                                 cudaStream_t st);

}  // namespace cupbr_b200
