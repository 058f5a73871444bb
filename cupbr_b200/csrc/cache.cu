// Radiance-cache training samples from the path tracer's own training paths
// (see cache.hpp).  A training path records, at every hit of depth k, the
// throughput T_k that reached the vertex and the radiance L_<k gathered
// before it; once the wavefront is finished its final radiance L gives the
// radiance leaving vertex k along the path, (L - L_<k) / T_k: the vertex's
// emission, direct light and everything further along the path, i.e. what a
// cached path ending at that vertex with the same bounces left needs from
// the cache.
#include "cache.hpp"

#include "wavefront.cuh"

namespace cupbr_b200 {

namespace {

constexpr float RC_MIN_THROUGHPUT = 1e-4f;  // vertices reached with less (any channel) are not used

// One thread per (training path, depth).
__global__ void k_rc_collect(PTFrame F, Workspace W, CacheFrame C, float4* __restrict__ samples,
                             uint32_t* __restrict__ n_samples, uint32_t capacity, uint32_t n_train) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tidx = g / F.max_depth, k = g - tidx * F.max_depth;
    bool push = false;
    float4 v[RC_REC];
    if (tidx < n_train && k < C.tcount[tidx]) {
        const float4* src = C.tverts + RC_REC * ((size_t)tidx * F.max_depth + k);
#pragma unroll
        for (int i = 0; i < (int)RC_REC; ++i) v[i] = src[i];
        const f3 T = xyz(v[4]);
        if (v[0].w != 0.0f && fminf(T.x, fminf(T.y, T.z)) >= RC_MIN_THROUGHPUT) {
            const uint32_t pid = tidx * C.train_stride + C.train_phase;
            const f3 L = xyz(W.radiance[pid]);
            const f3 before = mk(v[2].w, v[3].w, v[4].w);
            const f3 out = mk(fmaxf(L.x - before.x, 0.0f) / T.x, fmaxf(L.y - before.y, 0.0f) / T.y,
                              fmaxf(L.z - before.z, 0.0f) / T.z);
            v[0].w = 0.0f;
            v[2].w = (float)(F.max_depth - k);
            v[3].w = 0.0f;
            v[4] = f4(out, 1.0f);
            push = true;
        }
    }
    const uint32_t s = claim_slot(push, n_samples);
    if (push && s < capacity) {
        float4* dst = samples + RC_REC * (size_t)s;
#pragma unroll
        for (int i = 0; i < (int)RC_REC; ++i) dst[i] = v[i];
    }
}

}  // namespace

cudaError_t rc_collect(const PTFrame& F, const Workspace& W, const CacheFrame& C, float4* samples, uint32_t* n_samples,
                       uint32_t capacity, cudaStream_t st) {
    if (C.train_stride == 0 || F.n_paths <= C.train_phase) return cudaSuccess;
    const uint32_t n_train = (F.n_paths - C.train_phase + C.train_stride - 1) / C.train_stride;
    const uint64_t threads = (uint64_t)n_train * F.max_depth;
    k_rc_collect<<<(uint32_t)((threads + 255) / 256), 256, 0, st>>>(F, W, C, samples, n_samples, capacity, n_train);
    return cudaGetLastError();
}

}  // namespace cupbr_b200
