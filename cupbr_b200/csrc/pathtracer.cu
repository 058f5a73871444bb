// Wavefront NEE path tracer (RenderingMethod::PATHTRACER).
//
// One render() = one sample per pixel folded into the running mean, exactly
// as PBRendering::pathtracing / pathtracer_kernel_nee
// (lib/src/Renderer/PathTracer.cu:97-169, 260-276) define it, but organised
// as a wavefront over compact SoA queues instead of one thread per path:
//
//   k_camera      tea<4> seed, 2 jitter draws, camera ray  -> ray queue[0]
//   per bounce b < maxTraceDepth:
//     k_extend    closest hit for ray queue[b]              -> hit buffer
//     k_shade     emission, light / env selection, NEE ray, RR, BSDF sample
//                                                           -> shadow queue,
//                                                              ray queue[b+1]
//     k_connect   any hit for the shadow queue; visible contributions are
//                 added to the path's radiance
//   k_accumulate  running mean into the HDR image (PathTracer.cu:162-168)
//
// Every path keeps its own LCG state, consumed in the reference's order per
// bounce: light pick (1), light or env-BSDF sample, RR (1, if enabled), BSDF
// sample.  A path whose throughput becomes exactly zero (back-facing hit,
// PathTracer.cu:37-41) stops early: its remaining contributions are all
// zero and its RNG stream is private, so no other pixel changes.
//
// Queue slots are claimed with warp-aggregated atomics (one atomicAdd per
// warp, ballot + popc for the lane offsets); the traversal kernels are
// persistent and fetch 32 rays per warp from a global counter, with the top
// of the BVH staged in shared memory.
#include "pathtracer.hpp"

#include "cache.hpp"
#include "nvtx_range.hpp"
#include "path_shade.cuh"
#include "shading.cuh"
#include "trace.cuh"
#include "wavefront.cuh"

namespace cupbr_b200 {

namespace {

__global__ void k_camera(PTFrame F, Workspace W) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot == 0) W.ctr[CTR_RAYS + 0] = F.n_paths;
    if (slot >= F.n_paths) return;
    const uint32_t fr = slot / F.pixels;
    const uint32_t tid = slot_pixel(slot - fr * F.pixels, F.width, F.height);
    const uint32_t p = fr * F.pixels + tid;  // path
    // TracingDetail.h:15-30 (index2pixel: KernelHelperDetail.h:13-20)
    uint32_t seed = tea4(tid, F.frame_index + fr);
    const uint32_t py = tid / F.width;
    const uint32_t px = tid - F.width * py;
    float jx = rnd(seed);
    float jy = rnd(seed);
    const float rx = 2.0f * (((float)px + jx) / (float)F.width - 0.5f);
    const float ry = 2.0f * (((float)py + jy) / (float)F.height - 0.5f);
    f3 wp = F.cam_pos + F.cam_z + rx * F.cam_x + ry * F.cam_y;
    f3 d = normalize(wp - F.cam_pos);
    float4* q = W.rays[0] + 3 * (size_t)slot;
    q[0] = f4(F.cam_pos, __uint_as_float(p));
    q[1] = f4(d, __uint_as_float(seed));
    q[2] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    W.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Closest hit of ray queue[depth] into the hit buffer (persistent, dynamic
// fetch; see persistent_trace).
template <bool COUNT>
__global__ void __launch_bounds__(PT_TRACE_THREADS) k_extend(DeviceScene S, Workspace W, uint32_t depth,
                                                              uint32_t min_count) {
    if (W.ctr[CTR_RAYS + depth] < min_count) return;  // cached frames: left to k_tail
    extern __shared__ float4 s_nodes[];
    persistent_trace<false, COUNT>(S, W.rays[depth & 1], 3, W.ctr[CTR_RAYS + depth], &W.ctr[CTR_EFETCH + depth],
                                   W.smem_nodes, s_nodes, &W.err[ERR_STACK], W.stats + STAT_EXT_NODES,
                                   [&](uint32_t idx, const TravState& s) {
                                       W.hits[idx] = make_float2(s.t_best, __int_as_float(s.best_prim));
                                   });
}

// Closest hit of the camera-ray queue (depth 0) as warp packets: k_camera
// fills 32 consecutive slots from one 8x4 pixel tile (packet_trace).
__global__ void __launch_bounds__(PT_TRACE_THREADS) k_extend_camera(DeviceScene S, Workspace W, uint32_t min_count) {
    if (W.ctr[CTR_RAYS + 0] < min_count) return;  // cached frames: left to k_tail
    extern __shared__ float4 s_nodes[];
    packet_trace(S, W.rays[0], 3, W.ctr[CTR_RAYS + 0], &W.ctr[CTR_EFETCH + 0], W.smem_nodes, s_nodes,
                 &W.err[ERR_STACK], [&](uint32_t idx, const TravState& s) {
                     W.hits[idx] = make_float2(s.t_best, __int_as_float(s.best_prim));
                 });
}

// Shadow queue of depth: visible contributions are added to the path
// radiance (TracingDetail.h:181-182 visible -> PathTracer.cu:66-72).
// Held at 8 blocks per SM (64 registers) like the closest-hit kernels, which
// set the traversal grid: unconstrained it takes 72 registers, 7 blocks fit
// and the eighth of the grid starts late.
template <bool COUNT>
__global__ void __launch_bounds__(PT_TRACE_THREADS, 8) k_connect(DeviceScene S, Workspace W, uint32_t depth) {
    extern __shared__ float4 s_nodes[];
    persistent_trace<true, COUNT>(S, W.shadow, 3, W.ctr[CTR_SHADOW + depth], &W.ctr[CTR_CFETCH + depth], W.smem_nodes,
                                  s_nodes, &W.err[ERR_STACK], W.stats + STAT_SH_NODES,
                                  [&](uint32_t idx, const TravState& s) {
                                      if (s.hit) return;
                                      const float4* e = W.shadow + 3 * (size_t)idx;
                                      const float4 c = __ldg(e + 2);
                                      const uint32_t pid = __float_as_uint(__ldg(e + 1).w);
                                      float4 r = W.radiance[pid];
                                      r.x += c.x; r.y += c.y; r.z += c.z;
                                      W.radiance[pid] = r;
                                  });
}

// 4 blocks of 256 per SM (64 registers; measured faster than the
// unconstrained 92 registers at 2 blocks, despite a few spilled bytes).
template <bool CACHE, bool PHYS>
__global__ void __launch_bounds__(256, 4) k_shade(DeviceScene S, PTFrame F, Workspace W, uint32_t depth, CacheFrame C) {
    shade_stage<CACHE, PHYS>(S, F, W, depth, C);
}

// Tail of a frame: once ray queue[depth] holds fewer than C.tail_threshold
// rays, one thread carries each of them through its closest hit, shading,
// shadow ray and the following bounces until the path ends (the same
// shading code and traversal results as the wavefront stages, in the same
// order per path).  The wavefront kernels of this and later depths then find
// their queues empty.
template <bool CACHE, bool PHYS>
__global__ void __launch_bounds__(128) k_tail(DeviceScene S, PTFrame F, Workspace W, uint32_t depth, CacheFrame C) {
    const uint32_t count = W.ctr[CTR_RAYS + depth];
    if (count == 0 || count >= C.tail_threshold) return;
    const float4* __restrict__ q = W.rays[depth & 1];
    TraceCounters tc;
    bool overflow = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        float4 q0 = q[3 * (size_t)i], q1 = q[3 * (size_t)i + 1], q2 = q[3 * (size_t)i + 2];
        for (uint32_t d = depth;; ++d) {
            float t;
            int32_t prim;
            uint32_t key;
            trace_scene_rt(false, false, S, nullptr, 0, xyz(q0), xyz(q1), 0.0f, t, prim, key, overflow, tc);
            ShadeOut so;
            shade_one<CACHE, PHYS>(S, F, W, C, d, q0, q1, q2, make_float2(t, __int_as_float(prim)), so);
            if (so.sh) {
                float ts;
                int32_t ps;
                uint32_t ks;
                const bool hit = trace_scene_rt(true, false, S, nullptr, 0, xyz(so.s0), xyz(so.s1), so.s0.w, ts, ps,
                                                ks, overflow, tc);
                if (!hit) {
                    const uint32_t pid = __float_as_uint(so.s1.w);
                    float4 r = W.radiance[pid];
                    r.x += so.s2.x; r.y += so.s2.y; r.z += so.s2.z;
                    W.radiance[pid] = r;
                }
            }
            if (CACHE && so.q) {
                const uint32_t qs = atomicAdd(C.n_queries, 1u);
#pragma unroll
                for (int k = 0; k < (int)RC_REC; ++k) C.queries[(size_t)k * C.query_stride + qs] = so.cq[k];
            }
            if (!so.ext) break;
            q0 = so.e0;
            q1 = so.e1;
            q2 = so.e2;
        }
    }
    if (overflow) atomicAdd(&W.err[ERR_STACK], 1u);
}

// Folds the wavefront's frames into the running mean in frame order
// (PathTracer.cu:162-168), so a batch of frames equals that many render()s.
__global__ void k_accumulate(PTFrame F, Workspace W, float* __restrict__ img) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= F.pixels) return;
    float* o = img + 3 * (size_t)tid;
    f3 acc = mk(o[0], o[1], o[2]);
    for (uint32_t fr = 0; fr < F.frames; ++fr) {
        const f3 rad = xyz(W.radiance[(size_t)fr * F.pixels + tid]);
        const uint32_t f = F.frame_index + fr;
        if (f > 0) {
            const float a = 1.0f / ((float)f + 1.0f);
            acc = (1.0f - a) * acc + a * rad;
        } else {
            acc = rad;
        }
    }
    o[0] = acc.x; o[1] = acc.y; o[2] = acc.z;
}

// Closest hit (dist == nullptr) or visibility for caller rays; directions are
// normalized as the Ray constructor does (RayDetail.h:8-14).
__global__ void k_trace_rays(DeviceScene S, uint32_t n, const float* __restrict__ o, const float* __restrict__ d,
                             const float* __restrict__ dist, float* __restrict__ t_out, int32_t* __restrict__ prim_out,
                             uint32_t* __restrict__ key_out, int32_t* __restrict__ vis_out, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 org = mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
    f3 dir = normalize(mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
    float t;
    int32_t prim;
    uint32_t key;
    bool overflow = false;
    TraceCounters tc;
    if (dist) {
        bool occ = trace_scene<true, false>(S, nullptr, 0, org, dir, dist[i], t, prim, key, overflow, tc);
        vis_out[i] = occ ? 0 : 1;
    } else {
        trace_scene<false, false>(S, nullptr, 0, org, dir, 0.0f, t, prim, key, overflow, tc);
        t_out[i] = t;
        prim_out[i] = prim;
        key_out[i] = key;
    }
    if (overflow) atomicAdd(err, 1u);
}

}  // namespace

// ---------------------------------------------------------------- host ---

cudaError_t launch_trace_rays(const DeviceScene& S, uint32_t n, const float* o, const float* d, const float* dist,
                              float* t_out, int32_t* prim_out, uint32_t* key_out, int32_t* vis_out, uint32_t* err,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_trace_rays<<<(n + 127) / 128, 128, 0, st>>>(S, n, o, d, dist, t_out, prim_out, key_out, vis_out, err);
    return cudaGetLastError();
}

cudaError_t pt_launch_extend(const DeviceScene& S, const Workspace& W, uint32_t depth, int num_sms, cudaStream_t st,
                             uint32_t min_count, bool count) {
    const int smem = (int)(std::min(S.n_nodes, W.smem_nodes) * BVH_NODE_BYTES);
    if (count) k_extend<true><<<num_sms * W.trace_blocks_per_sm, PT_TRACE_THREADS, smem, st>>>(S, W, depth, min_count);
    else k_extend<false><<<num_sms * W.trace_blocks_per_sm, PT_TRACE_THREADS, smem, st>>>(S, W, depth, min_count);
    return cudaGetLastError();
}

cudaError_t pt_launch_extend_camera(const DeviceScene& S, const Workspace& W, int num_sms, cudaStream_t st,
                                    uint32_t min_count) {
    const int smem = (int)(std::min(S.n_nodes, W.smem_nodes) * BVH_NODE_BYTES);
    k_extend_camera<<<num_sms * W.trace_blocks_per_sm, PT_TRACE_THREADS, smem, st>>>(S, W, min_count);
    return cudaGetLastError();
}

cudaError_t pt_launch_tail(const DeviceScene& S, const PTFrame& F, const Workspace& W, const CacheFrame& C,
                           uint32_t depth, int num_sms, cudaStream_t st) {
    if (C.tail_threshold == 0) return cudaSuccess;
    const uint32_t blocks = std::min<uint32_t>((C.tail_threshold + 127) / 128, (uint32_t)num_sms * 16u);
    k_tail<true, false><<<blocks, 128, 0, st>>>(S, F, W, depth, C);
    return cudaGetLastError();
}

cudaError_t pt_launch_connect(const DeviceScene& S, const Workspace& W, uint32_t depth, int num_sms, cudaStream_t st,
                              bool count) {
    const int smem = (int)(std::min(S.n_nodes, W.smem_nodes) * BVH_NODE_BYTES);
    if (count) k_connect<true><<<num_sms * W.trace_blocks_per_sm, PT_TRACE_THREADS, smem, st>>>(S, W, depth);
    else k_connect<false><<<num_sms * W.trace_blocks_per_sm, PT_TRACE_THREADS, smem, st>>>(S, W, depth);
    return cudaGetLastError();
}

cudaError_t pt_launch_shade(const DeviceScene& S, const PTFrame& F, const Workspace& W, uint32_t depth, int num_sms,
                            cudaStream_t st) {
    if (F.estimator) k_shade<false, true><<<num_sms * 8, 256, 0, st>>>(S, F, W, depth, CacheFrame{});
    else k_shade<false, false><<<num_sms * 8, 256, 0, st>>>(S, F, W, depth, CacheFrame{});
    return cudaGetLastError();
}

cudaError_t pt_shade_cached(const DeviceScene& S, const PTFrame& F, const Workspace& W, const CacheFrame& C,
                            uint32_t depth, int num_sms, cudaStream_t st) {
    k_shade<true, false><<<num_sms * 8, 256, 0, st>>>(S, F, W, depth, C);
    return cudaGetLastError();
}

cudaError_t pt_launch_camera(const PTFrame& F, const Workspace& W, cudaStream_t st) {
    k_camera<<<(F.n_paths + 255) / 256, 256, 0, st>>>(F, W);
    return cudaGetLastError();
}

cudaError_t pt_launch_accumulate(const PTFrame& F, const Workspace& W, float* img, cudaStream_t st) {
    k_accumulate<<<(F.pixels + 255) / 256, 256, 0, st>>>(F, W, img);
    return cudaGetLastError();
}

int pt_occupancy_blocks(int smem_bytes) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_extend<false>, PT_TRACE_THREADS, smem_bytes);
    return b > 0 ? b : 1;
}

cudaError_t pt_render_frame(const DeviceScene& S, const PTFrame& F, const Workspace& W, float* img, cudaStream_t st,
                            int num_sms, bool count_stats, cudaEvent_t* ev, uint32_t tail_paths) {
    NvtxRange nvtx_("pt wavefront");
    cudaError_t e = cudaMemsetAsync(W.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st);
    if (e != cudaSuccess) return e;
    const uint32_t nb = (F.n_paths + 255) / 256;
    int ei = 0;
    auto mark = [&]() { if (ev) cudaEventRecord(ev[ei++], st); };
    mark();
    k_camera<<<nb, 256, 0, st>>>(F, W);
    mark();
    const int smem = (int)(std::min(S.n_nodes, W.smem_nodes) * BVH_NODE_BYTES);
    const int trace_blocks = num_sms * W.trace_blocks_per_sm;
    const int shade_blocks = num_sms * 8;
    // instrumented frames count every ray's traversal: no tail there
    CacheFrame T{};
    T.tail_threshold = count_stats ? 0u : tail_paths;
    const uint32_t tail_blocks = std::min<uint32_t>((T.tail_threshold + 127) / 128, (uint32_t)num_sms * 16u);
    for (uint32_t d = 0; d < F.max_depth; ++d) {
        if (T.tail_threshold) {
            if (F.estimator) k_tail<false, true><<<tail_blocks, 128, 0, st>>>(S, F, W, d, T);
            else k_tail<false, false><<<tail_blocks, 128, 0, st>>>(S, F, W, d, T);
        }
        if (count_stats) k_extend<true><<<trace_blocks, PT_TRACE_THREADS, smem, st>>>(S, W, d, 0u);
        else if (d == 0) k_extend_camera<<<trace_blocks, PT_TRACE_THREADS, smem, st>>>(S, W, T.tail_threshold);
        else k_extend<false><<<trace_blocks, PT_TRACE_THREADS, smem, st>>>(S, W, d, T.tail_threshold);
        mark();
        if (F.estimator) k_shade<false, true><<<shade_blocks, 256, 0, st>>>(S, F, W, d, T);
        else k_shade<false, false><<<shade_blocks, 256, 0, st>>>(S, F, W, d, T);
        mark();
        if (count_stats) k_connect<true><<<trace_blocks, PT_TRACE_THREADS, smem, st>>>(S, W, d);
        else k_connect<false><<<trace_blocks, PT_TRACE_THREADS, smem, st>>>(S, W, d);
        mark();
    }
    if (img) k_accumulate<<<(F.pixels + 255) / 256, 256, 0, st>>>(F, W, img);
    mark();
    return cudaGetLastError();
}

}  // namespace cupbr_b200
