// Batched multi-view path tracing (see batch.hpp): wavefront planning, the
// batch camera and accumulation kernels; the traversal and shading stages
// are the path tracer's own.
#include "batch.hpp"

#include <algorithm>

#include "wavefront.cuh"

namespace cupbr_b200 {

namespace {

// Last segment whose first path / pixel is <= i (segments are sorted).
template <bool PIX>
__device__ __forceinline__ uint32_t find_segment(const BatchSegment* __restrict__ segs, uint32_t nseg, uint32_t i) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t start = PIX ? __ldg(&segs[mid].pix0) : __ldg(&segs[mid].path0);
        if (start <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// TracingDetail.h:15-30 camera rays of every path of the wavefront (as the
// path tracer's k_camera, per view; the queue goes by 8x4 pixel tiles).
__global__ void k_batch_camera(const BatchSegment* __restrict__ segs, uint32_t nseg,
                               const BatchView* __restrict__ views, Workspace W, uint32_t n_paths) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot == 0) W.ctr[CTR_RAYS + 0] = n_paths;
    if (slot >= n_paths) return;
    const BatchSegment sg = segs[find_segment<false>(segs, nseg, slot)];
    const BatchView& v = views[sg.view];
    const uint32_t pixels = v.width * v.height;
    const uint32_t local = slot - sg.path0;
    const uint32_t fr = local / pixels;
    // slots in 8x4 pixel tiles (slot_pixel), traced as warp packets
    const uint32_t tid = slot_pixel(local - fr * pixels, v.width, v.height);
    const uint32_t p = sg.path0 + fr * pixels + tid;  // path
    uint32_t seed = tea4(tid, v.frame0 + sg.first + fr);
    const uint32_t py = tid / v.width, px = tid - v.width * py;
    const float jx = rnd(seed);
    const float jy = rnd(seed);
    const float rx = 2.0f * (((float)px + jx) / (float)v.width - 0.5f);
    const float ry = 2.0f * (((float)py + jy) / (float)v.height - 0.5f);
    const f3 wp = v.cam_pos + v.cam_z + rx * v.cam_x + ry * v.cam_y;
    const f3 d = normalize(wp - v.cam_pos);
    float4* q = W.rays[0] + 3 * (size_t)slot;
    q[0] = f4(v.cam_pos, __uint_as_float(p));
    q[1] = f4(d, __uint_as_float(seed));
    q[2] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    W.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Folds each segment's frames into its view's running mean in frame order
// (PathTracer.cu:162-168), one thread per pixel of every segment.
__global__ void k_batch_accumulate(const BatchSegment* __restrict__ segs, uint32_t nseg,
                                   const BatchView* __restrict__ views, Workspace W, uint32_t n_pixels) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pixels) return;
    const BatchSegment sg = segs[find_segment<true>(segs, nseg, i)];
    const BatchView& v = views[sg.view];
    const uint32_t pixels = v.width * v.height;
    const uint32_t tid = i - sg.pix0;
    float* o = v.img + 3 * (size_t)tid;
    f3 acc = mk(o[0], o[1], o[2]);
    for (uint32_t fr = 0; fr < sg.frames; ++fr) {
        const f3 rad = xyz(W.radiance[(size_t)sg.path0 + (size_t)fr * pixels + tid]);
        const uint32_t f = v.frame0 + sg.first + fr;
        if (f > 0) {
            const float a = 1.0f / ((float)f + 1.0f);
            acc = (1.0f - a) * acc + a * rad;
        } else {
            acc = rad;
        }
    }
    o[0] = acc.x;
    o[1] = acc.y;
    o[2] = acc.z;
}

}  // namespace

void batch_plan(const std::vector<uint32_t>& view_scene, const std::vector<BatchView>& views, uint32_t n_scenes,
                uint32_t capacity, std::vector<BatchWave>& waves, std::vector<BatchSegment>& segs) {
    waves.clear();
    segs.clear();
    for (uint32_t sc = 0; sc < n_scenes; ++sc) {
        BatchWave w{sc, (uint32_t)segs.size(), 0, 0, 0};
        auto close = [&]() {
            if (w.nseg) waves.push_back(w);
            w = BatchWave{sc, (uint32_t)segs.size(), 0, 0, 0};
        };
        for (uint32_t v = 0; v < (uint32_t)views.size(); ++v) {
            if (view_scene[v] != sc) continue;
            const uint32_t pixels = views[v].width * views[v].height;
            uint32_t done = 0;
            while (done < views[v].spp) {
                uint32_t room = (capacity - w.n_paths) / pixels;
                if (room == 0) {
                    close();
                    room = std::max(1u, capacity / pixels);
                }
                const uint32_t take = std::min(room, views[v].spp - done);
                segs.push_back(BatchSegment{w.n_paths, w.n_pixels, v, done, take});
                ++w.nseg;
                w.n_paths += take * pixels;
                w.n_pixels += pixels;
                done += take;
            }
        }
        close();
    }
}

cudaError_t batch_record_wave(const DeviceScene& S, const BatchWave& w, const BatchSegment* dsegs,
                              const BatchView* dviews, const Workspace& W, uint32_t max_depth, int num_sms,
                              cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(W.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st);
    if (e != cudaSuccess) return e;
    k_batch_camera<<<(w.n_paths + 255) / 256, 256, 0, st>>>(dsegs + w.seg0, w.nseg, dviews, W, w.n_paths);
    PTFrame F{};
    F.max_depth = max_depth;
    F.use_rr = 0;
    for (uint32_t d = 0; d < max_depth; ++d) {
        e = d == 0 ? pt_launch_extend_camera(S, W, num_sms, st) : pt_launch_extend(S, W, d, num_sms, st);
        if (e != cudaSuccess) return e;
        if ((e = pt_launch_shade(S, F, W, d, num_sms, st)) != cudaSuccess) return e;
        if ((e = pt_launch_connect(S, W, d, num_sms, st)) != cudaSuccess) return e;
    }
    k_batch_accumulate<<<(w.n_pixels + 255) / 256, 256, 0, st>>>(dsegs + w.seg0, w.nseg, dviews, W, w.n_pixels);
    return cudaGetLastError();
}

}  // namespace cupbr_b200
