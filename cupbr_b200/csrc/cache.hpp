// Learned radiance cache: a 96-64-64-64-64-64-16 ReLU MLP (5 hidden layers
// of 64, FP16 weights and activations, FP32 accumulation in tensor memory)
// that maps a path vertex to the radiance leaving it, trained online on
// radiance the path tracer itself produces and queried to end cached paths
// early.  The reference has no counterpart; the path tracer it shortens is
// PathTracer.cu:20-169.
//
// Matrices live in shared memory (and, for the weights, in global memory) as
// 8 x 8 "core matrices" of 128 contiguous bytes: element (r, c) of an R x C
// matrix sits at rc_tiled(r, c, C).  With that one layout a matrix serves as
// a K-major operand when its columns are the contraction and as an MN-major
// operand when its rows are, so the forward, input-gradient and
// weight-gradient products read the same activations and weights without
// transposed copies.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "pathtracer.hpp"

namespace cupbr_b200 {

constexpr uint32_t RC_IN = 96;       // encoded input width (84 used, zero padded)
constexpr uint32_t RC_HID = 64;      // hidden width
constexpr uint32_t RC_OUT = 16;      // output rows of the last layer (3 used: RGB)
constexpr uint32_t RC_LAYERS = 6;    // weight matrices
constexpr uint32_t RC_TILE = 128;    // rows (vertices) per tensor-core tile
constexpr uint32_t RC_WEIGHTS = 64 * 96 + 4 * 64 * 64 + 16 * 64;  // tiled elements (23552)
constexpr uint32_t RC_PARAMS = 64 * 96 + 4 * 64 * 64 + 3 * 64;    // trainable weights (22720)
constexpr uint32_t RC_REC = 5;       // float4 per query / training record
constexpr uint32_t RC_BANDS = 12;    // frequency bands of the position encoding
constexpr float RC_BOUNCE_NORM = 16.0f;  // remaining bounces enter the network as min(r, 16) / 16

__host__ __device__ constexpr uint32_t rc_in(uint32_t l) { return l == 0 ? RC_IN : RC_HID; }
__host__ __device__ constexpr uint32_t rc_out(uint32_t l) { return l == RC_LAYERS - 1 ? RC_OUT : RC_HID; }
__host__ __device__ constexpr uint32_t rc_woff(uint32_t l) { return l == 0 ? 0u : 64u * 96u + 4096u * (l - 1u); }
// element (r, c) of an R x C matrix stored as 8 x 8 core matrices, row groups outer
__host__ __device__ constexpr uint32_t rc_tiled(uint32_t r, uint32_t c, uint32_t C) {
    return (((r >> 3) * (C >> 3) + (c >> 3)) << 6) + ((r & 7u) << 3) + (c & 7u);
}

// Scene box that positions are normalised to before the frequency encoding.
struct RcBounds {
    f3 lo, inv_ext;
};

// Query and training record (RC_REC float4):
//   [0] position, w: path index (queries)
//   [1] direction towards the previous vertex, w: roughness
//   [2] shading normal, w: bounces the path tracer had left at the vertex
//       (max depth - depth): the cache learns the truncated estimator
//   [3] diffuse albedo, w: -
//   [4] queries: path throughput; samples: target radiance, w: weight (0 or 1)
//
// Network state on the device.  master / adam_m / adam_v / w16 / grad use the
// tiled order of rc_tiled per layer (offsets rc_woff).
struct RcNet {
    float* master = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    __half* w16 = nullptr;      // FP16 copy of master (training)
    float* ema = nullptr;       // exponential moving average of master
    __half* w16_ema = nullptr;  // FP16 copy of the bias-corrected average (inference)
    float* grad = nullptr;      // mean gradient of the last step
    float* partials = nullptr;  // per training CTA weight gradients
    float* loss = nullptr;      // [0] relative L2 sum, [1] weighted samples (last step)
    uint32_t* err = nullptr;    // [0] CTAs whose tensor-core wait ran out of time; [1] of those, CTAs
                                // whose second wait (for the MMAs still in flight) ran out as well
    uint32_t partial_ctas = 0;
    uint32_t wait_probe_ns = 0;  // test hook: inference CTAs wait this long on a barrier nothing arrives on
};

// Loss of a training sample (RGB, weight w, prediction y, target t):
//   RC_LOSS_RELATIVE  w (y - t)^2 / (y^2 + 0.01), y^2 held constant
//   RC_LOSS_L2        w (y - t)^2
enum RcLoss : uint32_t { RC_LOSS_RELATIVE = 0, RC_LOSS_L2 = 1 };

struct RcAdam {
    float lr, beta1, beta2, eps;
    uint32_t step;     // 1-based step about to be taken
    float ema_decay;   // weight average for inference (0: inference uses the latest weights)
    uint32_t loss;     // RcLoss
};

// Inference reads w16 (the caller passes N.w16_ema or N.w16 as `weights`).
// Raw inference: out[i] = network(records[i]) (RGB, w = 0).
cudaError_t rc_infer(const RcNet& N, const __half* weights, const RcBounds& B, const float4* recs, uint32_t n,
                     float4* out, int num_sms, cudaStream_t st);
// Cached-path inference: radiance[path] += throughput * max(network, 0) for
// the *count queries (count read on the device, at most capacity), whose
// records are component-major with stride capacity (CacheFrame::queries).
cudaError_t rc_infer_queries(const RcNet& N, const __half* weights, const RcBounds& B, const float4* recs,
                             const uint32_t* count, uint32_t capacity, float4* radiance, int num_sms, cudaStream_t st);
// One Adam step on n samples (n a multiple of RC_TILE, at most
// RC_TILE * N.partial_ctas) with the loss A.loss summed over the RGB
// channels, mean over the weighted samples.  Row j of the step reads samples[base + j] when count is
// null, else one of the min(*count, capacity) collected samples: a stride
// over them when there are at least `total`, cycling otherwise.
cudaError_t rc_train_step(const RcNet& N, const RcBounds& B, const float4* samples, const uint32_t* count,
                          uint32_t capacity, uint32_t base, uint32_t total, uint32_t n, const RcAdam& A,
                          cudaStream_t st);

// Per-wavefront state of a cached frame.  Path p of the wavefront is a
// training path when train_stride != 0 and p % train_stride == train_phase;
// its index among them is p / train_stride.
struct CacheFrame {
    // RC_REC float4 per cached path end, component-major (structure of
    // arrays): float4 k of query q at queries[k * query_stride + q], so the
    // shading stage's writes and the inference kernel's reads coalesce
    float4* queries;
    uint32_t query_stride;  // the wavefront's paths (the most queries it can make)
    uint32_t* n_queries;    // device counter
    float4* tverts;         // RC_REC float4 per (training path, depth)
    uint32_t* tcount;       // per training path: depths recorded
    uint32_t cache_depth;   // first depth whose hit the cache answers
    uint32_t train_stride;  // 0: no training paths
    uint32_t train_phase;
    uint32_t specular;      // != 0: mirror and glass vertices beyond cache_depth are answered too
    uint32_t train_end;     // training paths end in a cache query at depths >= train_end (0: never)
    uint32_t tail_threshold;  // a ray queue with fewer rays goes to pt_launch_tail (0: never)
};
// The path tracer's shading stage with the cache hooks (pathtracer.cu).
cudaError_t pt_shade_cached(const DeviceScene& S, const PTFrame& F, const Workspace& W, const CacheFrame& C,
                            uint32_t depth, int num_sms, cudaStream_t st);
// Per-path tail (pathtracer.cu): when ray queue[depth] holds fewer than
// C.tail_threshold rays, one thread per ray traces the rest of its path.
cudaError_t pt_launch_tail(const DeviceScene& S, const PTFrame& F, const Workspace& W, const CacheFrame& C,
                           uint32_t depth, int num_sms, cudaStream_t st);
// Training samples from the recorded vertices of one wavefront's training
// paths: target = (final radiance - radiance before the vertex) / throughput,
// appended at *n_samples (at most capacity).
cudaError_t rc_collect(const PTFrame& F, const Workspace& W, const CacheFrame& C, float4* samples,
                       uint32_t* n_samples, uint32_t capacity, cudaStream_t st);

}  // namespace cupbr_b200
