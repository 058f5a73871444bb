// Batched multi-view path tracing (see batch.hpp): wavefront planning, the
// batch camera and accumulation kernels; the traversal and shading stages
// are the path tracer's own.
#include "batch.hpp"

#include <algorithm>

#include "path_shade.cuh"
#include "trace.cuh"
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

// TracingDetail.h:15-30 camera ray of queue slot `slot` of the wavefront
// (as the path tracer's k_camera, per view; the queue goes by 8x4 pixel tiles).
__device__ __forceinline__ void batch_camera_slot(const BatchSegment* __restrict__ segs, uint32_t nseg,
                                                  const BatchView* __restrict__ views, const Workspace& W,
                                                  uint32_t slot) {
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

__global__ void k_batch_camera(const BatchSegment* __restrict__ segs, uint32_t nseg,
                               const BatchView* __restrict__ views, Workspace W, uint32_t n_paths) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot == 0) W.ctr[CTR_RAYS + 0] = n_paths;
    if (slot >= n_paths) return;
    batch_camera_slot(segs, nseg, views, W, slot);
}

// Folds pixel i of the wavefront's segments into its view's running mean in
// frame order (PathTracer.cu:162-168).  NC as qload.
template <bool NC>
__device__ __forceinline__ void batch_accumulate_pixel(const BatchSegment* __restrict__ segs, uint32_t nseg,
                                                       const BatchView* __restrict__ views, const Workspace& W,
                                                       uint32_t i) {
    const BatchSegment sg = segs[find_segment<true>(segs, nseg, i)];
    const BatchView& v = views[sg.view];
    const uint32_t pixels = v.width * v.height;
    const uint32_t tid = i - sg.pix0;
    float* o = v.img + 3 * (size_t)tid;
    f3 acc = NC ? mk(o[0], o[1], o[2]) : mk(__ldcg(o), __ldcg(o + 1), __ldcg(o + 2));
    for (uint32_t fr = 0; fr < sg.frames; ++fr) {
        const float4* rp = &W.radiance[(size_t)sg.path0 + (size_t)fr * pixels + tid];
        const f3 rad = xyz(NC ? *rp : __ldcg(rp));
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

__global__ void k_batch_accumulate(const BatchSegment* __restrict__ segs, uint32_t nseg,
                                   const BatchView* __restrict__ views, Workspace W, uint32_t n_pixels) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pixels) return;
    batch_accumulate_pixel<true>(segs, nseg, views, W, i);
}

// ---- one cooperative launch over every wavefront of the batch ----------

// Grid-wide barrier of the cooperative kernel (all blocks resident): the
// last block to arrive releases the others by bumping the generation.  Every
// wait is bounded (limit_ns, BATCH_BARRIER_NS by default): a block that gives up sets `abort`,
// which releases the others, and every block returns; the host reads the
// abort flag as an error.  The fences order each block's writes before its
// arrival and the released blocks' later loads after the release.
constexpr uint64_t BATCH_BARRIER_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ uint64_t batch_gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_barrier(BatchBarrier* gb, uint32_t nblocks, uint64_t limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile uint32_t* gen = &gb->gen;
        volatile uint32_t* abort_flag = &gb->abort;
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const uint64_t t0 = batch_gtimer();
            while (*gen == g) {
                if (*abort_flag) { ok = 0; break; }
                if (batch_gtimer() - t0 > limit_ns) {
                    atomicExch(&gb->abort, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        if (*abort_flag) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// The batch's wavefronts in one launch: per wavefront the camera stage, per
// depth the closest-hit (camera packets at depth 0), shading and shadow-ray
// stages, and the accumulation, each stage over the whole grid with a grid
// barrier after it.  Same stage code as the wavefront mode's kernels, with
// state loads that bypass the non-coherent caches (qload<false>).
// probe_ns > 0 (test hook): block 0 leaves before the first barrier, which
// the other blocks then wait on for probe_ns before they give up, set the
// abort flag and return (a barrier that times out, with no fault).
__global__ void __launch_bounds__(256, 2) k_batch_coop(const DeviceScene* __restrict__ scenes,
                                                       const BatchWave* __restrict__ waves, uint32_t n_waves,
                                                       const BatchSegment* __restrict__ segs,
                                                       const BatchView* __restrict__ views, Workspace W,
                                                       uint32_t max_depth, BatchBarrier* gb, uint64_t probe_ns) {
    constexpr int WORDS = (int)(sizeof(DeviceScene) / sizeof(uint32_t));
    __shared__ DeviceScene S;
    const uint32_t nblocks = gridDim.x;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
    const uint64_t limit_ns = probe_ns ? probe_ns : BATCH_BARRIER_NS;
    if (probe_ns && blockIdx.x == 0) return;
    PTFrame F{};
    F.max_depth = max_depth;
    F.use_rr = 0;
    const CacheFrame C{};
    for (uint32_t wi = 0; wi < n_waves; ++wi) {
        const BatchWave wv = waves[wi];
        const uint32_t* src = reinterpret_cast<const uint32_t*>(scenes + wv.scene);
        for (int k = (int)threadIdx.x; k < WORDS; k += (int)blockDim.x)
            reinterpret_cast<uint32_t*>(&S)[k] = __ldg(&src[k]);
        for (uint32_t i = gtid; i < CTR_TOTAL; i += gsize) W.ctr[i] = (i == CTR_RAYS + 0) ? wv.n_paths : 0u;
        for (uint32_t slot = gtid; slot < wv.n_paths; slot += gsize)
            batch_camera_slot(segs + wv.seg0, wv.nseg, views, W, slot);
        if (!grid_barrier(gb, nblocks, limit_ns)) return;
        for (uint32_t d = 0; d < max_depth; ++d) {
            const uint32_t nrays = __ldcg(&W.ctr[CTR_RAYS + d]);
            auto hit = [&](uint32_t idx, const TravState& s) {
                W.hits[idx] = make_float2(s.t_best, __int_as_float(s.best_prim));
            };
            if (d == 0)
                packet_trace<false>(S, W.rays[0], 3, nrays, &W.ctr[CTR_EFETCH + 0], 0u, nullptr, &W.err[ERR_STACK],
                                    hit);
            else
                persistent_trace<false, false, false>(S, W.rays[d & 1], 3, nrays, &W.ctr[CTR_EFETCH + d], 0u, nullptr,
                                                      &W.err[ERR_STACK], W.stats, hit);
            if (!grid_barrier(gb, nblocks, limit_ns)) return;
            shade_stage<false, false, false>(S, F, W, d, C);
            if (!grid_barrier(gb, nblocks, limit_ns)) return;
            const uint32_t nsh = __ldcg(&W.ctr[CTR_SHADOW + d]);
            persistent_trace<true, false, false>(S, W.shadow, 3, nsh, &W.ctr[CTR_CFETCH + d], 0u, nullptr,
                                                 &W.err[ERR_STACK], W.stats, [&](uint32_t idx, const TravState& s) {
                                                     if (s.hit) return;
                                                     const float4* e = W.shadow + 3 * (size_t)idx;
                                                     const float4 c = __ldcg(e + 2);
                                                     const uint32_t pid = __float_as_uint(__ldcg(e + 1).w);
                                                     float4 r = __ldcg(&W.radiance[pid]);
                                                     r.x += c.x; r.y += c.y; r.z += c.z;
                                                     W.radiance[pid] = r;
                                                 });
            if (!grid_barrier(gb, nblocks, limit_ns)) return;
        }
        for (uint32_t i = gtid; i < wv.n_pixels; i += gsize)
            batch_accumulate_pixel<false>(segs + wv.seg0, wv.nseg, views, W, i);
        if (!grid_barrier(gb, nblocks, limit_ns)) return;
    }
}

// The persistent batch kernel (batch_launch_persistent).  Each warp copies
// its item's DeviceScene record into shared memory (the record is read on
// every node visit and shading call) and keeps it while consecutive items
// share the scene.  PACKET: the camera rays of a frame (the warp's 8x4
// tile) find their closest hits as one warp packet (packet_closest), the
// later bounces one thread per path; otherwise every ray is traced on its
// own.  Both give the same hits.
// 512 / THREADS resident blocks (16 warps per SM, 128 registers a thread):
// the compiler's own choice at 64 and 128 threads spills ~150 bytes.
template <int THREADS, bool PACKET>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) k_batch_persistent(const DeviceScene* __restrict__ scenes,
                                                              const BatchView* __restrict__ views,
                                                              const BatchItem* __restrict__ items, uint32_t n_items,
                                                              uint32_t* counter, uint32_t max_depth, uint32_t* err) {
    constexpr int WARPS = THREADS / 32;
    constexpr int WORDS = (int)(sizeof(DeviceScene) / sizeof(uint32_t));
    static_assert(sizeof(DeviceScene) % sizeof(uint32_t) == 0, "DeviceScene copied word by word");
    __shared__ DeviceScene s_scene[WARPS];
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    DeviceScene& S = s_scene[wid];
    uint32_t cur_scene = 0xFFFFFFFFu;
    bool overflow = false;
    TraceCounters tc;
    PTFrame F{};
    F.max_depth = max_depth;
    F.use_rr = 0;
    const CacheFrame C{};
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(counter, 1u);
        it = __shfl_sync(full, it, 0);
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const BatchView v = views[bi.view];
        if (v.scene != cur_scene) {
            __syncwarp();
            const uint32_t* src = reinterpret_cast<const uint32_t*>(scenes + v.scene);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&S);
            for (int k = (int)lane; k < WORDS; k += 32) dst[k] = __ldg(&src[k]);
            __syncwarp();
            cur_scene = v.scene;
        }
        const uint32_t pixels = v.width * v.height;
        const uint32_t slot = bi.slot0 + lane;
        const bool valid = slot < pixels;
        if (!PACKET && !valid) continue;
        const uint32_t tid = valid ? slot_pixel(slot, v.width, v.height) : 0u;
        const uint32_t py = tid / v.width, px = tid - v.width * py;
        float* o = v.img + 3 * (size_t)tid;
        f3 acc = valid ? mk(o[0], o[1], o[2]) : splat(0.0f);
        for (uint32_t fr = 0; fr < v.spp; ++fr) {
            const uint32_t f = v.frame0 + fr;
            // camera ray (TracingDetail.h:15-30, as k_batch_camera)
            uint32_t seed = tea4(tid, f);
            const float jx = rnd(seed);
            const float jy = rnd(seed);
            const float rx = 2.0f * (((float)px + jx) / (float)v.width - 0.5f);
            const float ry = 2.0f * (((float)py + jy) / (float)v.height - 0.5f);
            const f3 wp = v.cam_pos + v.cam_z + rx * v.cam_x + ry * v.cam_y;
            float4 q0 = f4(v.cam_pos, __uint_as_float(tid));
            float4 q1 = f4(normalize(wp - v.cam_pos), __uint_as_float(seed));
            float4 q2 = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            float t = 0.0f;
            int32_t prim = HIT_NONE;
            if (PACKET) {
                TravState ts;
                int32_t st_ref[CUPBR_STACK_SIZE];
                float st_t[CUPBR_STACK_SIZE];
                packet_closest(S, nullptr, 0, xyz(q0), xyz(q1), valid, ts, st_ref, st_t, overflow);
                t = ts.t_best;
                prim = ts.best_prim;
            }
            if (valid) {
                f3 rad = splat(0.0f);
                for (uint32_t d = 0;; ++d) {
                    if (!PACKET || d > 0) {
                        uint32_t key;
                        trace_scene_rt(false, false, S, nullptr, 0, xyz(q0), xyz(q1), 0.0f, t, prim, key, overflow,
                                       tc);
                    }
                    ShadeOut so;
                    shade_core<false, false>(S, F, C, d, q0, q1, q2, make_float2(t, __int_as_float(prim)), rad, so);
                    if (so.sh) {
                        float ts;
                        int32_t ps;
                        uint32_t ks;
                        if (!trace_scene_rt(true, false, S, nullptr, 0, xyz(so.s0), xyz(so.s1), so.s0.w, ts, ps, ks,
                                            overflow, tc))
                            rad += xyz(so.s2);
                    }
                    if (!so.ext) break;
                    q0 = so.e0;
                    q1 = so.e1;
                    q2 = so.e2;
                }
                // running mean (PathTracer.cu:162-168)
                if (f > 0) {
                    const float a = 1.0f / ((float)f + 1.0f);
                    acc = (1.0f - a) * acc + a * rad;
                } else {
                    acc = rad;
                }
            }
            if (PACKET) __syncwarp();
        }
        if (valid) {
            o[0] = acc.x;
            o[1] = acc.y;
            o[2] = acc.z;
        }
    }
    if (overflow) atomicAdd(err, 1u);
}

// Adjoint of the persistent kernel's frames with respect to the scenes'
// albedo textures (batch_launch_backward): each thread replays its path of
// every frame from the path's seed -- the same camera ray, traversal and
// shading, so the same vertices -- and records, at each textured Lambert
// vertex, the texel and the radiance gathered before that vertex's light
// term.  Every radiance term from that light term on carries the texel's
// albedo exactly once per channel (Lambert sampling does not depend on the
// albedo; Russian roulette is off), so its derivative with respect to the
// texel is (path radiance - radiance before) / albedo, scattered with
// weight dLoss/dImage / (frame0 + spp) (the running mean's weight of one
// frame).
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) k_batch_backward(const DeviceScene* __restrict__ scenes,
                                                            const BatchView* __restrict__ views,
                                                            const BatchItem* __restrict__ items, uint32_t n_items,
                                                            uint32_t* counter, uint32_t max_depth,
                                                            const float* const* __restrict__ grad_img,
                                                            float* const* __restrict__ grad_tex, uint32_t* err) {
    constexpr int WARPS = THREADS / 32;
    constexpr int WORDS = (int)(sizeof(DeviceScene) / sizeof(uint32_t));
    __shared__ DeviceScene s_scene[WARPS];
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    DeviceScene& S = s_scene[wid];
    uint32_t cur_scene = 0xFFFFFFFFu;
    bool overflow = false;
    TraceCounters tc;
    PTFrame F{};
    F.max_depth = max_depth;
    F.use_rr = 0;
    const CacheFrame C{};
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(counter, 1u);
        it = __shfl_sync(full, it, 0);
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const BatchView v = views[bi.view];
        if (v.scene != cur_scene) {
            __syncwarp();
            const uint32_t* src = reinterpret_cast<const uint32_t*>(scenes + v.scene);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&S);
            for (int k = (int)lane; k < WORDS; k += 32) dst[k] = __ldg(&src[k]);
            __syncwarp();
            cur_scene = v.scene;
        }
        float* gt = grad_tex[v.scene];
        const float* gi = grad_img[bi.view];
        const uint32_t pixels = v.width * v.height;
        const uint32_t slot = bi.slot0 + lane;
        if (!gt || !gi || !S.tex || slot >= pixels) continue;
        const uint32_t tid = slot_pixel(slot, v.width, v.height);
        const float inv_n = 1.0f / ((float)v.frame0 + (float)v.spp);
        const f3 g = mk(gi[3 * (size_t)tid], gi[3 * (size_t)tid + 1], gi[3 * (size_t)tid + 2]) * inv_n;
        if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f) continue;
        const uint32_t py = tid / v.width, px = tid - v.width * py;
        for (uint32_t fr = 0; fr < v.spp; ++fr) {
            const uint32_t f = v.frame0 + fr;
            uint32_t seed = tea4(tid, f);
            const float jx = rnd(seed);
            const float jy = rnd(seed);
            const float rx = 2.0f * (((float)px + jx) / (float)v.width - 0.5f);
            const float ry = 2.0f * (((float)py + jy) / (float)v.height - 0.5f);
            const f3 wp = v.cam_pos + v.cam_z + rx * v.cam_x + ry * v.cam_y;
            float4 q0 = f4(v.cam_pos, __uint_as_float(tid));
            float4 q1 = f4(normalize(wp - v.cam_pos), __uint_as_float(seed));
            float4 q2 = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            f3 rad = splat(0.0f);
            int32_t rec_t[BATCH_BWD_MAX_DEPTH];
            f3 rec_c[BATCH_BWD_MAX_DEPTH];
            uint32_t nrec = 0;
            for (uint32_t d = 0;; ++d) {
                float t;
                int32_t prim;
                uint32_t key;
                trace_scene_rt(false, false, S, nullptr, 0, xyz(q0), xyz(q1), 0.0f, t, prim, key, overflow, tc);
                ShadeOut so;
                shade_core<false, false>(S, F, C, d, q0, q1, q2, make_float2(t, __int_as_float(prim)), rad, so);
                if (so.texel >= 0 && nrec < BATCH_BWD_MAX_DEPTH) {
                    rec_t[nrec] = so.texel;
                    rec_c[nrec] = rad;
                    ++nrec;
                }
                if (so.sh) {
                    float ts;
                    int32_t ps;
                    uint32_t ks;
                    if (!trace_scene_rt(true, false, S, nullptr, 0, xyz(so.s0), xyz(so.s1), so.s0.w, ts, ps, ks,
                                        overflow, tc))
                        rad += xyz(so.s2);
                }
                if (!so.ext) break;
                q0 = so.e0;
                q1 = so.e1;
                q2 = so.e2;
            }
            for (uint32_t k = 0; k < nrec; ++k) {
                const f3 a = xyz(S.tex[rec_t[k]]);
                const f3 after = rad - rec_c[k];
                float* o = gt + 3 * (size_t)rec_t[k];
                if (a.x > 0.0f && after.x != 0.0f) atomicAdd(o, g.x * after.x / a.x);
                if (a.y > 0.0f && after.y != 0.0f) atomicAdd(o + 1, g.y * after.y / a.y);
                if (a.z > 0.0f && after.z != 0.0f) atomicAdd(o + 2, g.z * after.z / a.z);
            }
        }
    }
    if (overflow) atomicAdd(err, 1u);
}

}  // namespace

void batch_items(const std::vector<BatchView>& views, const std::vector<uint32_t>& scene_nodes,
                 std::vector<BatchItem>& items) {
    items.clear();
    std::vector<uint32_t> order(views.size());
    for (uint32_t i = 0; i < (uint32_t)views.size(); ++i) order[i] = i;
    auto cost = [&](uint32_t v) {
        return (double)views[v].spp * (double)std::max<uint32_t>(1u, scene_nodes[views[v].scene]);
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost(a) > cost(b); });
    for (uint32_t v : order) {
        const uint32_t pixels = views[v].width * views[v].height;
        for (uint32_t s0 = 0; s0 < pixels; s0 += 32u) items.push_back(BatchItem{v, s0});
    }
}

int batch_persistent_occupancy(uint32_t threads, bool packet) {
    int b = 0;
    if (packet) {
        if (threads == 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<64, true>, 64, 0);
        else if (threads == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<256, true>, 256, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<128, true>, 128, 0);
    } else {
        if (threads == 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<64, false>, 64, 0);
        else if (threads == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<256, false>, 256, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_persistent<128, false>, 128, 0);
    }
    return b > 0 ? b : 1;
}

int batch_coop_occupancy() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_coop, 256, 0);
    return b;
}

cudaError_t batch_launch_coop(const DeviceScene* scenes, const BatchWave* waves, uint32_t n_waves,
                              const BatchSegment* segs, const BatchView* views, const Workspace& W,
                              uint32_t max_depth, uint32_t blocks_per_sm, int num_sms, BatchBarrier* gb,
                              cudaStream_t st, uint64_t probe_ns) {
    const int full = batch_coop_occupancy();
    if (full < 1) return cudaErrorCooperativeLaunchTooLarge;
    const uint32_t bps = blocks_per_sm ? std::min<uint32_t>(blocks_per_sm, (uint32_t)full) : (uint32_t)full;
    cudaError_t e = cudaMemsetAsync(gb, 0, sizeof(BatchBarrier), st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(bps * (uint32_t)num_sms);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    Workspace w = W;
    return cudaLaunchKernelEx(&cfg, k_batch_coop, scenes, waves, n_waves, segs, views, w, max_depth, gb, probe_ns);
}

cudaError_t batch_launch_backward(const DeviceScene* scenes, const BatchView* views, const BatchItem* items,
                                  uint32_t n_items, uint32_t* counter, uint32_t max_depth, const float* const* grad_img,
                                  float* const* grad_tex, uint32_t threads, uint32_t blocks_per_sm, int num_sms,
                                  uint32_t* err, cudaStream_t st) {
    if (max_depth > BATCH_BWD_MAX_DEPTH) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::max(1u, blocks_per_sm) * (uint32_t)num_sms;
    if (threads == 64)
        k_batch_backward<64><<<blocks, 64, 0, st>>>(scenes, views, items, n_items, counter, max_depth, grad_img,
                                                    grad_tex, err);
    else if (threads == 256)
        k_batch_backward<256><<<blocks, 256, 0, st>>>(scenes, views, items, n_items, counter, max_depth, grad_img,
                                                      grad_tex, err);
    else
        k_batch_backward<128><<<blocks, 128, 0, st>>>(scenes, views, items, n_items, counter, max_depth, grad_img,
                                                      grad_tex, err);
    return cudaGetLastError();
}

int batch_backward_occupancy(uint32_t threads) {
    int b = 0;
    if (threads == 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_backward<64>, 64, 0);
    else if (threads == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_backward<256>, 256, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_backward<128>, 128, 0);
    return b > 0 ? b : 1;
}

template <bool PACKET>
static void launch_persistent(uint32_t threads, uint32_t blocks, cudaStream_t st, const DeviceScene* scenes,
                              const BatchView* views, const BatchItem* items, uint32_t n_items, uint32_t* counter,
                              uint32_t max_depth, uint32_t* err) {
    if (threads == 64)
        k_batch_persistent<64, PACKET><<<blocks, 64, 0, st>>>(scenes, views, items, n_items, counter, max_depth, err);
    else if (threads == 256)
        k_batch_persistent<256, PACKET><<<blocks, 256, 0, st>>>(scenes, views, items, n_items, counter, max_depth, err);
    else
        k_batch_persistent<128, PACKET><<<blocks, 128, 0, st>>>(scenes, views, items, n_items, counter, max_depth, err);
}

cudaError_t batch_launch_persistent(const DeviceScene* scenes, const BatchView* views, const BatchItem* items,
                                    uint32_t n_items, uint32_t* counter, uint32_t max_depth, uint32_t threads,
                                    uint32_t blocks_per_sm, bool packet, int num_sms, uint32_t* err, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::max(1u, blocks_per_sm) * (uint32_t)num_sms;
    if (packet) launch_persistent<true>(threads, blocks, st, scenes, views, items, n_items, counter, max_depth, err);
    else launch_persistent<false>(threads, blocks, st, scenes, views, items, n_items, counter, max_depth, err);
    return cudaGetLastError();
}

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
