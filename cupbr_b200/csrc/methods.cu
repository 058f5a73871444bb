// RenderingMethod::VOLUME, GRADIENTDOMAIN and RAYTRACER.
//
// VOLUME (VolumeRenderer.cu:11-310) and the GDPT paths
// (GradientDomain.cu:110-246) run as wavefronts on the path tracer's
// persistent traversal kernels, with their own shading stages: a VOLUME
// path inside a VOLUME object only sees that object (the shading stage
// intersects it itself), and a GDPT shift path stops where its base path's
// vertex is invalid (base paths first, shift paths in a second wavefront).
// RAYTRACER is one thread per pixel over one out-of-line traversal.  The
// GDPT reconstruction (init_kernel + 50 optimization passes,
// GradientDomain.cu:248-350, 379-401) ping-pongs between two buffers instead
// of copying temp back each pass.  Arithmetic follows dev_common.cuh's
// contract, operation order the reference's.
#include "methods.hpp"

#include "nvtx_range.hpp"
#include "shading.cuh"
#include "trace.cuh"
#include "wavefront.cuh"

namespace cupbr_b200 {

namespace {

__device__ __forceinline__ float comp(f3 v, uint32_t i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ f3 vexp(f3 v) { return mk(expf(v.x), expf(v.y), expf(v.z)); }

// Tracing::launchRay (TracingDetail.h:15-45)
__device__ __forceinline__ void camera_ray(const PTFrame& F, uint32_t px, uint32_t py, bool jitter, uint32_t& seed,
                                           f3& o, f3& d) {
    float jx = jitter ? rnd(seed) : 0.0f;
    float jy = jitter ? rnd(seed) : 0.0f;
    const float rx = 2.0f * (((float)px + jx) / (float)F.width - 0.5f);
    const float ry = 2.0f * (((float)py + jy) / (float)F.height - 0.5f);
    f3 wp = F.cam_pos + F.cam_z + rx * F.cam_x + ry * F.cam_y;
    o = F.cam_pos;
    d = normalize(wp - F.cam_pos);
}

struct Surf {
    float t;
    f3 P, N;
    int32_t obj;
};

// Traversal counters of an instrumented launch (on = false: not counted).
struct MCount {
    bool on = false;
    TraceCounters ext, sh;
    uint32_t ext_rays = 0, sh_rays = 0;
};

// Result of one traversal (trace_call).
struct RtOut {
    float t;
    int32_t prim;
    uint32_t nodes, tris;
    bool hit, ovf;
};

// Every closest-hit and shadow query of the per-pixel kernels goes through
// this one out-of-line copy of the traversal: their loops trace from several
// places, and inlined copies of the loop at each of them left most warps
// stalled on instruction fetch.  S must be a __grid_constant__ kernel
// parameter (or global memory): its address is taken without a local copy.
__device__ __noinline__ RtOut trace_call(bool any, bool count, const DeviceScene& S, f3 o, f3 d, float t_limit) {
    RtOut r;
    TraceCounters c;
    uint32_t key;
    r.ovf = false;
    r.hit = trace_scene_rt(any, count, S, nullptr, 0, o, d, t_limit, r.t, r.prim, key, r.ovf, c);
    r.nodes = c.nodes;
    r.tris = c.tris;
    return r;
}

__device__ __forceinline__ bool closest(const DeviceScene& S, f3 o, f3 d, Surf& h, bool& ovf, MCount& mc) {
    const RtOut r = trace_call(false, mc.on, S, o, d, 0.0f);
    ovf |= r.ovf;
    if (mc.on) {
        mc.ext.nodes += r.nodes;
        mc.ext.tris += r.tris;
        mc.ext_rays += 1u;
    }
    const float t = r.t;
    const int32_t prim = r.prim;
    h.t = t;
    if (prim == HIT_NONE) return false;
    h.P = o + t * d;
    hit_normal(S, prim, h.P, h.N, h.obj);
    return true;
}

__device__ __forceinline__ bool visible(const DeviceScene& S, float dist, f3 o, f3 d, bool& ovf, MCount& mc) {
    const RtOut r = trace_call(true, mc.on, S, o, d, dist);
    ovf |= r.ovf;
    if (mc.on) {
        mc.sh.nodes += r.nodes;
        mc.sh.tris += r.tris;
        mc.sh_rays += 1u;
    }
    return !r.hit;
}

__device__ __forceinline__ MatView object_material(const DeviceScene& S, int32_t obj) {
    return load_material(S.materials, __float_as_int(__ldg(&S.objects[obj].hi).w));
}

// Light or env-BSDF sample of directIllumination (PathTracer.cu:43-62 and its
// copies in VolumeRenderer.cu / GradientDomain.cu).
__device__ __forceinline__ f3 sample_nee(const DeviceScene& S, const MatView& m, uint32_t& seed, f3 P, f3 inc, f3 N,
                                         f3& ldir, float& dist) {
    const uint32_t L = S.n_lights, use_env = S.env_w > 0 ? 1u : 0u;
    uint32_t ls = (uint32_t)(rnd(seed) * (float)(L + use_env));
    if (ls != L) return sample_light(S.lights, ls, seed, P, ldir, dist);
    float4 s = sample_direction(m, seed, inc, N);
    ldir = xyz(s);
    dist = __int_as_float(0x7f800000);
    return use_env ? env_lookup(S, ldir) / s.w : splat(0.0f);
}

// ---- VOLUME as a wavefront ------------------------------------------------
// The path state of the reference's per-pixel loop (VolumeRenderer.cu:11-87)
// lives in the path tracer's ray records:
// (origin, path), (direction, seed), (throughput, tag), tag = 0 for a path
// outside every VOLUME object, object + 1 for a path inside one.  Paths
// outside go to the front of the next ray queue (their closest hits come
// from the path tracer's persistent traversal kernels), paths inside to its
// back (counted in CTR_VOL_INSIDE): they only see their own object, which
// the shading stage intersects itself (trace_object).  A light term whose
// visibility the reference tests inline becomes a shadow-queue entry with
// its contribution, added by the path tracer's k_connect if unoccluded.
// Each path adds at most one term per depth, in depth order, so the running
// sums are the per-pixel kernel's.
constexpr uint32_t CTR_VOL_INSIDE = CTR_MVERT;  // the medium's vertex counters, unused by VOLUME frames

// Class of an outside entry's hit for ordering the shading work: 0 miss,
// 1 VOLUME interface, 2 diffuse (Lambert, Phong), 3 GGX, 4 mirror or glass.
__device__ __forceinline__ uint32_t vol_class(const DeviceScene& S, float2 h) {
    const int32_t prim = __float_as_int(h.y);
    if (prim == HIT_NONE) return 0u;
    const uint32_t slot = prim_slot(prim);
    int32_t obj;
    switch (prim_type(prim)) {
        case 0: obj = __float_as_int(__ldg(&S.tris[3 * (size_t)slot + 1]).w); break;
        case 1: obj = __float_as_int(__ldg(&S.spheres[2 * (size_t)slot + 1]).z); break;
        case 2: obj = __ldg(&S.quad_obj[slot]); break;
        default: obj = __float_as_int(__ldg(&S.planes[2 * (size_t)slot + 1]).w); break;
    }
    const int type = (int)__ldg(&S.materials[__float_as_int(__ldg(&S.objects[obj].hi).w)].e).w;
    return type == 5 ? 1u : type == 4 ? 3u : (type == 2 || type == 3) ? 4u : 2u;
}

// The body of the reference's depth loop (VolumeRenderer.cu:88-310) for one
// queue entry.
__global__ void __launch_bounds__(256, 2) k_vol_shade(const __grid_constant__ DeviceScene S, PTFrame F, Workspace W,
                                                      uint32_t depth) {
    const uint32_t n_out = W.ctr[CTR_RAYS + depth], n_in = W.ctr[CTR_VOL_INSIDE + depth];
    const uint32_t n = n_out + n_in;
    const float4* __restrict__ q = W.rays[depth & 1];
    float4* __restrict__ qn = W.rays[(depth + 1) & 1];
    const bool last = depth + 1 >= F.max_depth;
    const uint32_t L = S.n_lights, use_env = S.env_w > 0 ? 1u : 0u;
    const float nl = (float)(L + use_env);
    const f3 scene_ss = xyz(S.vol_sigma_s), scene_sa = xyz(S.vol_sigma_a);
    const float scene_g = S.vol_sigma_s.w;
    // each chunk of 256 entries is shaded in class order (misses, VOLUME
    // interfaces, diffuse, GGX, mirror / glass, paths inside an object), so
    // most warps run one branch of the bounce
    constexpr uint32_t NC = 6;
    __shared__ uint32_t s_cnt[8][NC];
    __shared__ uint32_t s_idx[256];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    for (uint32_t c0 = blockIdx.x * 256u; c0 < n; c0 += gridDim.x * 256u) {
        const uint32_t mine = c0 + threadIdx.x;
        uint32_t cls = NC;  // past the end
        if (mine < n) cls = mine >= n_out ? NC - 1 : vol_class(S, __ldg(&W.hits[mine]));
        uint32_t rank = 0;
#pragma unroll
        for (uint32_t k = 0; k < NC; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, cls == k);
            if (cls == k) rank = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) s_cnt[wid][k] = __popc(m);
        }
        __syncthreads();
        if (cls < NC) {
            uint32_t base = 0;
            for (uint32_t k = 0; k < cls; ++k)
                for (uint32_t w = 0; w < 8; ++w) base += s_cnt[w][k];
            for (uint32_t w = 0; w < wid; ++w) base += s_cnt[w][cls];
            s_idx[base + rank] = mine;
        }
        __syncthreads();
        const uint32_t i = threadIdx.x < n - c0 ? s_idx[threadIdx.x] : 0xFFFFFFFFu;
        bool push_sh = false, push_next = false, next_inside = false;
        float4 sh0, sh1, sh2, r0, r1, r2;
        if (i < n) {
            const uint32_t slot = i < n_out ? i : F.n_paths - 1 - (i - n_out);
            const float4 q0 = __ldg(&q[3 * (size_t)slot]), q1 = __ldg(&q[3 * (size_t)slot + 1]);
            const float4 q2 = __ldg(&q[3 * (size_t)slot + 2]);
            const f3 o = xyz(q0), d = xyz(q1);
            const uint32_t pid = __float_as_uint(q0.w);
            uint32_t seed = __float_as_uint(q1.w);
            f3 rw = xyz(q2);
            const uint32_t tag = __float_as_uint(q2.w);
            bool inside = tag != 0u;
            int32_t obj_index = inside ? (int32_t)(tag - 1u) : 0;
            f3 ray_start = splat(0.0f), out_dir = splat(0.0f);
            bool next_valid = false;
            Surf g;
            bool hit;
            if (inside) {
                hit = trace_object(S, obj_index, o, d, g.t, g.N);
                if (hit) {
                    g.P = o + g.t * d;
                    g.obj = obj_index;
                }
            } else {
                const float2 h = __ldg(&W.hits[slot]);
                g.t = h.x;
                const int32_t prim = __float_as_int(h.y);
                hit = prim != HIT_NONE;
                if (hit) {
                    g.P = o + g.t * d;
                    hit_normal(S, prim, g.P, g.N, g.obj);
                }
            }
            const f3 inc = -1.0f * d;
            if (!hit) {
                if (use_env) {
                    float4 r = W.radiance[pid];
                    const f3 e = rw * env_lookup(S, d);
                    r.x += e.x; r.y += e.y; r.z += e.z;
                    W.radiance[pid] = r;
                }
            } else {
                const MatView m = object_material(S, g.obj);
                f3 vss = scene_ss, vsa = scene_sa;
                float vg = scene_g;
                if (inside) {
                    const MatView im = object_material(S, obj_index);
                    vss = im.sigma_s;
                    vsa = im.sigma_a;
                    vg = im.g;
                }
                bool handled = false, stop = false;
                {
                    const f3 st = vsa + vss;
                    const uint32_t ch = (uint32_t)(rnd(seed) * 3.0f);
                    if (!feq0(comp(st, ch))) {
                        const float t = -logf(1.0f - rnd(seed)) / comp(st, ch);
                        if (t < g.t) {
                            handled = true;
                            const f3 Pe = o + t * d;
                            const float sp = comp(vss, ch) / comp(st, ch);
                            if (rnd(seed) < sp) {
                                float pdf = 0.0f;
                                for (uint32_t k = 0; k < 3; ++k) pdf += comp(st, k) * expf(-1.0f * comp(st, k) * t);
                                pdf /= 3.0f;
                                rw = rw * vss / sp * vexp(-1.0f * st * t) / pdf;
                                f3 ldir;
                                float dist;
                                const f3 lrad = sample_nee(S, m, seed, Pe, inc, g.N, ldir, dist);
                                f3 att = splat(1.0f);
                                f3 so = Pe + 0.001f * ldir;
                                if (inside) {
                                    float te;
                                    f3 Ne;
                                    f3 ePs = Pe;
                                    if (!trace_object(S, obj_index, Pe, normalize(ldir), te, Ne)) te = 0.0f;
                                    else ePs = Pe + te * normalize(ldir);
                                    att = vexp(-1.0f * st * te) * hg_phase(vg, -dot(inc, ldir));
                                    so = ePs + 0.001f * ldir;
                                    dist -= te;
                                } else if (F.estimator) {
                                    att = splat(hg_phase(vg, -dot(inc, ldir)));
                                }
                                const f3 sst = scene_sa + scene_ss;
                                const f3 c = nl * vexp(-1.0f * sst * fminf(dist, 100000000.0f)) * att * lrad * rw;
                                push_sh = true;
                                sh0 = f4(so, dist);
                                sh1 = f4(normalize(ldir), __uint_as_float(pid));
                                sh2 = f4(c, 0.0f);
                                const float4 shg = sample_hg(vg, -1.0f * inc, seed);
                                out_dir = xyz(shg);
                                ray_start = Pe;
                                next_valid = true;
                            } else {
                                rw = splat(0.0f);
                            }
                        } else {
                            float pdf = 0.0f;
                            for (uint32_t k = 0; k < 3; ++k) pdf += expf(-comp(st, k) * g.t);
                            pdf /= 3.0f;
                            rw = rw * vexp(-1.0f * st * g.t) / pdf;
                            ray_start = g.P;
                        }
                    }
                }
                if (!handled) {
                    if (m.type == 5) {  // VOLUME interface (VolumeRenderer.cu:269-278)
                        out_dir = xyz(sample_direction(m, seed, inc, g.N));
                        ray_start = g.P;
                        const bool refl = dot(inc, g.N) * dot(out_dir, g.N) > 0.0f;
                        inside = refl ? inside : !inside;
                        obj_index = g.obj;
                        next_valid = true;
                    } else {
                        if (m.type != 3 && dot(g.N, inc) <= 0.0f) {
                            rw = splat(0.0f);
                        } else {
                            f3 ldir;
                            float dist;
                            const f3 lrad = sample_nee(S, m, seed, g.P, inc, g.N, ldir, dist);
                            const f3 c = nl * fmaxf(0.0f, dot(g.N, ldir)) *
                                         vexp(-1.0f * (vss + vsa) * fminf(dist, 100000000.0f)) *
                                         brdf(m, inc, ldir, g.N) * lrad * rw;
                            push_sh = true;
                            sh0 = f4(g.P + 0.001f * ldir, dist);
                            sh1 = f4(normalize(ldir), __uint_as_float(pid));
                            sh2 = f4(c, 0.0f);
                        }
                        const float4 sd = sample_direction(m, seed, inc, g.N);
                        const f3 dir = xyz(sd);
                        if (!(norm(dir) == 0.0f)) {
                            rw = rw * fabsf(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / sd.w;
                            out_dir = dir;
                            ray_start = g.P;
                            next_valid = true;
                        }
                    }
                    if (F.use_rr) {
                        const float alpha = clampf(fmaxf(rw.x, fmaxf(rw.y, rw.z)), 0.0f, 1.0f);
                        if (rnd(seed) > alpha || feq0(alpha)) stop = true;
                        else rw = rw / alpha;
                    }
                }
                if (next_valid && !stop && !last) {
                    push_next = true;
                    next_inside = inside;
                    r0 = f4(ray_start + 0.001f * out_dir, __uint_as_float(pid));
                    r1 = f4(normalize(out_dir), __uint_as_float(seed));
                    r2 = f4(rw, __uint_as_float(inside ? (uint32_t)obj_index + 1u : 0u));
                }
            }
        }
        const uint32_t ss = claim_slot(push_sh, &W.ctr[CTR_SHADOW + depth]);
        const uint32_t so = claim_slot(push_next && !next_inside, &W.ctr[CTR_RAYS + depth + 1]);
        const uint32_t si = claim_slot(push_next && next_inside, &W.ctr[CTR_VOL_INSIDE + depth + 1]);
        if (push_sh) {
            float4* e = W.shadow + 3 * (size_t)ss;
            e[0] = sh0;
            e[1] = sh1;
            e[2] = sh2;
        }
        if (push_next) {
            float4* e = qn + 3 * (size_t)(next_inside ? F.n_paths - 1 - si : so);
            e[0] = r0;
            e[1] = r1;
            e[2] = r2;
        }
    }
}

// ---- GRADIENTDOMAIN paths as two wavefronts ------------------------------
// gdpt_kernel's five paths per interior pixel (GradientDomain.cu:160-246),
// for F.frames frames: first the
// base paths (queue slots over the interior in 8x4 tiles, frame by frame),
// which record per depth whether they hit (`valid`, one 64-bit mask per
// interior pixel and frame), then the four shift paths of every pixel whose
// base path hit at depth 0, each continued only while the base path's vertex
// at the next depth is valid.  With v = fr * n_int + j for interior pixel j
// (row major over the interior) of frame fr: base path id v, shift k (1..4)
// n_base + 4 v + k - 1, n_base = F.frames * n_int.  Emission is added in the
// shading stage, light terms by k_connect after it: per depth in the
// per-pixel kernel's order.

// Interior pixel j of the w x h image (j < (w - 2) (h - 2)) -> pixel index.
__device__ __forceinline__ uint32_t gd_pixel(uint32_t j, uint32_t w) {
    const uint32_t iw = w - 2u, iy = j / iw;
    return (iy + 1u) * w + (j - iy * iw) + 1u;
}

// The five camera rays of interior pixel j in frame fr of the batch
// (gdpt_kernel's seed chain); k = 0 base, 1..4 left, right, up, down.
__device__ __forceinline__ void gd_camera(const PTFrame& F, uint32_t j, uint32_t fr, uint32_t k, f3& o, f3& d,
                                          uint32_t& seed) {
    const uint32_t tid = gd_pixel(j, F.width);
    const uint32_t py = tid / F.width, px = tid - F.width * py;
    const int off[5][2] = {{0, 0}, {-1, 0}, {1, 0}, {0, 1}, {0, -1}};
    seed = tea4(tid, F.frame_index + fr);
    for (uint32_t c = 0; c <= k; ++c)
        camera_ray(F, (uint32_t)((int)px + off[c][0]), (uint32_t)((int)py + off[c][1]), true, seed, o, d);
}

// Base paths: slot s covers interior pixel slot_pixel(s % n_int) (8x4
// tiles) of frame s / n_int.
__global__ void k_gd_camera_base(PTFrame F, Workspace W, uint32_t n_int, uint64_t* __restrict__ valid) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n_base = F.frames * n_int;
    if (s == 0) W.ctr[CTR_RAYS + 0] = n_base;
    if (s >= n_base) return;
    const uint32_t fr = s / n_int;
    const uint32_t j = slot_pixel(s - fr * n_int, F.width - 2u, F.height - 2u);
    const uint32_t v = fr * n_int + j;
    f3 o, d;
    uint32_t seed;
    gd_camera(F, j, fr, 0, o, d, seed);
    float4* q = W.rays[0] + 3 * (size_t)s;
    q[0] = f4(o, __uint_as_float(v));
    q[1] = f4(d, __uint_as_float(seed));
    q[2] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    W.radiance[v] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    valid[v] = 0ull;
}

// Shift paths: t covers shift 1 + t % 4 of interior pixel
// slot_pixel((t % (4 n_int)) / 4) of frame t / (4 n_int); queued only where
// the base path hit at depth 0.
__global__ void k_gd_camera_shift(PTFrame F, Workspace W, uint32_t n_int, const uint64_t* __restrict__ valid) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n_base = F.frames * n_int;
    const bool in = t < 4u * n_base;
    uint32_t j = 0, k = 1, fr = 0, v = 0;
    bool want = false;
    if (in) {
        fr = t / (4u * n_int);
        const uint32_t l = t - fr * 4u * n_int;
        j = slot_pixel(l >> 2, F.width - 2u, F.height - 2u);
        k = 1u + (l & 3u);
        v = fr * n_int + j;
        want = (valid[v] & 1ull) != 0ull;
        W.radiance[n_base + 4u * v + k - 1u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    const uint32_t slot = claim_slot(want, &W.ctr[CTR_RAYS + 0]);
    if (!want) return;
    f3 o, d;
    uint32_t seed;
    gd_camera(F, j, fr, k, o, d, seed);
    float4* q = W.rays[0] + 3 * (size_t)slot;
    q[0] = f4(o, __uint_as_float(n_base + 4u * v + k - 1u));
    q[1] = f4(d, __uint_as_float(seed));
    q[2] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
}

// The body of collect_radiance's depth loop (GradientDomain.cu:110-158)
// for one queue entry.
template <bool SHIFT>
__global__ void __launch_bounds__(256, 2) k_gd_shade(const __grid_constant__ DeviceScene S, PTFrame F, Workspace W,
                                                     uint32_t depth, uint32_t n_base, uint64_t* __restrict__ valid) {
    const uint32_t n = W.ctr[CTR_RAYS + depth];
    const float4* __restrict__ q = W.rays[depth & 1];
    float4* __restrict__ qn = W.rays[(depth + 1) & 1];
    const bool last = depth + 1 >= F.max_depth;
    const uint32_t L = S.n_lights, use_env = S.env_w > 0 ? 1u : 0u;
    const float nl = (float)(L + use_env);
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        bool push_sh = false, push_next = false;
        float4 sh0, sh1, sh2, r0, r1, r2;
        if (i < n) {
            const float4 q0 = __ldg(&q[3 * (size_t)i]), q1 = __ldg(&q[3 * (size_t)i + 1]);
            const float4 q2 = __ldg(&q[3 * (size_t)i + 2]);
            const f3 o = xyz(q0), d = xyz(q1);
            const uint32_t pid = __float_as_uint(q0.w);
            uint32_t seed = __float_as_uint(q1.w);
            f3 rw = xyz(q2);
            const uint32_t j = SHIFT ? (pid - n_base) >> 2 : pid;  // v of the path's pixel and frame
            const float2 h = __ldg(&W.hits[i]);
            const int32_t prim = __float_as_int(h.y);
            if (prim == HIT_NONE) {
                if (use_env) {
                    float4 r = W.radiance[pid];
                    const f3 e = rw * env_lookup(S, d);
                    r.x += e.x; r.y += e.y; r.z += e.z;
                    W.radiance[pid] = r;
                }
            } else {
                Surf g;
                g.t = h.x;
                g.P = o + g.t * d;
                hit_normal(S, prim, g.P, g.N, g.obj);
                if (!SHIFT) valid[j] |= 1ull << depth;
                const f3 inc = -1.0f * d;
                const MatView m = object_material(S, g.obj);
                {
                    float4 r = W.radiance[pid];
                    const f3 e = rw * m.albedo_e;
                    r.x += e.x; r.y += e.y; r.z += e.z;
                    W.radiance[pid] = r;
                }
                if (m.type != 3 && dot(g.N, inc) <= 0.0f) {
                    rw = splat(0.0f);
                } else {
                    f3 ldir;
                    float dist;
                    const f3 lrad = sample_nee(S, m, seed, g.P, inc, g.N, ldir, dist);
                    const f3 c = nl * fmaxf(0.0f, dot(g.N, ldir)) * brdf(m, inc, ldir, g.N) * lrad * rw;
                    push_sh = true;
                    sh0 = f4(g.P + 0.001f * ldir, dist);
                    sh1 = f4(normalize(ldir), __uint_as_float(pid));
                    sh2 = f4(c, 0.0f);
                }
                const float4 sd = sample_direction(m, seed, inc, g.N);
                const f3 dir = xyz(sd);
                if (!(norm(dir) == 0.0f)) {
                    rw = rw * fabsf(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / sd.w;
                    bool go = !last;
                    if (SHIFT) go = go && !is_zero(rw) && ((__ldg(&valid[j]) >> (depth + 1)) & 1ull) != 0ull;
                    if (go) {
                        push_next = true;
                        r0 = f4(g.P + 0.01f * dir, __uint_as_float(pid));
                        r1 = f4(normalize(dir), __uint_as_float(seed));
                        r2 = f4(rw, 0.0f);
                    }
                }
            }
        }
        const uint32_t ss = claim_slot(push_sh, &W.ctr[CTR_SHADOW + depth]);
        const uint32_t sn = claim_slot(push_next, &W.ctr[CTR_RAYS + depth + 1]);
        if (push_sh) {
            float4* e = W.shadow + 3 * (size_t)ss;
            e[0] = sh0;
            e[1] = sh1;
            e[2] = sh2;
        }
        if (push_next) {
            float4* e = qn + 3 * (size_t)sn;
            e[0] = r0;
            e[1] = r1;
            e[2] = r2;
        }
    }
}

// gdpt_kernel's outputs from the five path radiances of frame fr of the batch:
// base and the four gradient estimates folded into their running means
// (interior pixels).
__global__ void k_gd_accumulate(PTFrame F, Workspace W, uint32_t n_int, uint32_t fr, float* __restrict__ base,
                                float* __restrict__ gxf, float* __restrict__ gxb, float* __restrict__ gyf,
                                float* __restrict__ gyb) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_int) return;
    const uint32_t tid = gd_pixel(j, F.width);
    const uint32_t v = fr * n_int + j, n_base = F.frames * n_int;
    f3 Lr[5];
    Lr[0] = xyz(W.radiance[v]);
    for (int k = 1; k < 5; ++k) Lr[k] = xyz(W.radiance[n_base + 4u * v + (uint32_t)k - 1u]);
    f3 out[5] = {Lr[0], 0.5f * (Lr[0] - Lr[1]), 0.5f * (Lr[2] - Lr[0]), 0.5f * (Lr[0] - Lr[4]),
                 0.5f * (Lr[3] - Lr[0])};
    float* bufs[5] = {base, gxf, gxb, gyf, gyb};
    const uint32_t f = F.frame_index + fr;
    const float a = 1.0f / ((float)f + 1.0f);
    for (int k = 0; k < 5; ++k) {
        float* qv = bufs[k] + 3 * (size_t)tid;
        f3 x = out[k];
        if (f > 0) x = (1.0f - a) * mk(qv[0], qv[1], qv[2]) + a * x;
        qv[0] = x.x; qv[1] = x.y; qv[2] = x.z;
    }
}

// Adds a wavefront's ray counts (closest-hit and shadow queues of every
// depth) to the instrumented frame's STAT_EXT_RAYS / STAT_SH_RAYS.
__global__ void k_ray_stats(Workspace W, uint32_t max_depth) {
    uint64_t e = 0, sh = 0;
    for (uint32_t d = 0; d < max_depth; ++d) {
        e += W.ctr[CTR_RAYS + d];
        sh += W.ctr[CTR_SHADOW + d];
    }
    W.stats[STAT_EXT_RAYS] += e;
    W.stats[STAT_SH_RAYS] += sh;
}

// init_kernel (GradientDomain.cu:248-273)
__global__ void k_gdpt_init(uint32_t w, uint32_t h, float* __restrict__ recon, const float* __restrict__ base,
                            const float* __restrict__ gxf, const float* __restrict__ gxb, const float* __restrict__ gyf,
                            const float* __restrict__ gyb, float* __restrict__ gx, float* __restrict__ gy) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= w * h) return;
    const size_t p = 3 * (size_t)tid;
    for (int c = 0; c < 3; ++c) recon[p + c] = base[p + c];
    const uint32_t y = tid / w, x = tid - w * y;
    if (x == 0 || y == 0 || x == w - 1 || y == h - 1) return;
    for (int c = 0; c < 3; ++c) {
        gx[p + c] = gxf[p + c] + gxb[p + c];
        gy[p + c] = gyf[p + c] + gyb[p + c];
    }
}

__device__ __forceinline__ float median4(float v0, float v1, float v2, float v3) {  // compute_median :275-301
    const float v[4] = {v0, v1, v2, v3};
    float med = 0.0f;
    uint32_t amin = 0, amax = 0;
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i) {
        med += v[i];
        if (v[i] < v[amin]) amin = i;
        if (v[i] > v[amax]) amax = i;
    }
    return (med - v[amin] - v[amax]) / 2.0f;
}

// optimization_kernel (GradientDomain.cu:303-350): src -> dst (interior).
// copy_border: the border pixels of dst take src's (see
// launch_gdpt_reconstruct).  Launched as a chain of programmatic dependent
// launches: each pass lets the next one be scheduled as soon as its own
// blocks start, and waits for the previous pass to complete (and its
// writes to be visible) before it reads anything, so the 50 short passes
// overlap their launch latencies instead of paying them one after another.
__global__ void k_gdpt_opt(uint32_t w, uint32_t h, const float* __restrict__ src, const float* __restrict__ gx,
                           const float* __restrict__ gy, float* __restrict__ dst, int copy_border) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= w * h) return;
    const uint32_t y = tid / w, x = tid - w * y;
    if (x == 0 || y == 0 || x == w - 1 || y == h - 1) {
        if (copy_border)
            for (int c = 0; c < 3; ++c) dst[3 * (size_t)tid + c] = src[3 * (size_t)tid + c];
        return;
    }
    const size_t p = tid, l = p - 1, r = p + 1, u = p + w, dn = p - w;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float v1 = src[3 * l + c] + gx[3 * l + c];
        const float v2 = src[3 * dn + c] + gy[3 * dn + c];
        const float v3 = src[3 * r + c] - gx[3 * p + c];
        const float v4 = src[3 * u + c] - gy[3 * p + c];
        dst[3 * p + c] = median4(v1, v2, v3, v4);
    }
}

// raytracing_kernel (RayTracer.cu:11-54): direct light from every light's
// position and intensity, no jitter, no accumulation.
__global__ void k_raytrace(const __grid_constant__ DeviceScene S, PTFrame F, float* __restrict__ img, uint32_t* err) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= F.n_paths) return;
    const uint32_t py = tid / F.width, px = tid - F.width * py;
    uint32_t seed = 0;
    f3 o, d;
    camera_ray(F, px, py, false, seed, o, d);
    bool ovf = false;
    MCount mc;
    Surf g;
    f3 rad = splat(0.0f);
    if (closest(S, o, d, g, ovf, mc)) {
        const f3 inc = normalize(F.cam_pos - g.P);
        const MatView m = object_material(S, g.obj);
        for (uint32_t i = 0; i < S.n_lights; ++i) {
            const f3 lp = xyz(__ldg(&S.lights[i].pos));
            const f3 ldir = normalize(lp - g.P);
            const f3 b = brdf(m, inc, ldir, g.N);
            const float dist = norm(g.P - lp);
            const f3 lrad = xyz(__ldg(&S.lights[i].I)) / (dist * dist);
            const float cosTerm = fmaxf(0.0f, dot(g.N, ldir));
            if (visible(S, dist, g.P - CUPBR_EPS * d, normalize(ldir), ovf, mc)) rad += b * lrad * cosTerm;
        }
    }
    if (ovf) atomicAdd(err, 1u);
    float* q = img + 3 * (size_t)tid;
    q[0] = rad.x; q[1] = rad.y; q[2] = rad.z;
}

}  // namespace

cudaError_t volume_render_frame(const DeviceScene& S, const PTFrame& F, const Workspace& W, float* img, cudaStream_t st,
                                int num_sms, bool count_stats) {
    NvtxRange nvtx_("volume wavefront");
    cudaError_t e = cudaMemsetAsync(W.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st);
    if (e != cudaSuccess) return e;
    if ((e = pt_launch_camera(F, W, st)) != cudaSuccess) return e;
    for (uint32_t d = 0; d < F.max_depth; ++d) {
        e = d == 0 && !count_stats ? pt_launch_extend_camera(S, W, num_sms, st)
                                   : pt_launch_extend(S, W, d, num_sms, st, 0u, count_stats);
        if (e != cudaSuccess) return e;
        k_vol_shade<<<num_sms * 8, 256, 0, st>>>(S, F, W, d);
        if ((e = pt_launch_connect(S, W, d, num_sms, st, count_stats)) != cudaSuccess) return e;
    }
    return img ? pt_launch_accumulate(F, W, img, st) : cudaGetLastError();
}

cudaError_t launch_gdpt_reconstruct(uint32_t w, uint32_t h, const float* base, const float* gxf, const float* gxb,
                                    const float* gyf, const float* gyb, float* gx, float* gy, float* temp, float* out,
                                    cudaStream_t st) {
    const uint32_t n = w * h;
    if (n == 0) return cudaSuccess;
    k_gdpt_init<<<(n + 255) / 256, 256, 0, st>>>(w, h, out, base, gxf, gxb, gyf, gyb, gx, gy);
    // GradientDomain.cu:392-401: 50 passes, each followed by a copy of the
    // whole of temp (its border included, which no pass writes) into the
    // output.  Here the passes alternate between the output and temp instead:
    // pass 0 reads the output with the border k_gdpt_init gave it; every
    // later pass must see temp's border there, so the passes that write the
    // output also copy temp's border into it.  The result lands in the output
    // after the even number of passes, as the reference's does.
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((n + 255) / 256);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    for (int i = 0; i < 50; ++i) {
        const float* src = (i & 1) ? temp : out;
        float* dst = (i & 1) ? out : temp;
        const float* cgx = gx;
        const float* cgy = gy;
        cudaError_t e = cudaLaunchKernelEx(&cfg, k_gdpt_opt, w, h, src, cgx, cgy, dst, i & 1);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t gdpt_trace_frames(const DeviceScene& S, const PTFrame& F, const Workspace& W, void* valid_scratch,
                              cudaStream_t st, int num_sms, bool count_stats) {
    NvtxRange nvtx_("gdpt wavefronts");
    const uint32_t w = F.width, h = F.height;
    if (w < 3 || h < 3) return cudaSuccess;  // no interior pixel, no path
    const uint32_t n_int = (w - 2) * (h - 2), n_base = F.frames * n_int;
    uint64_t* valid = reinterpret_cast<uint64_t*>(valid_scratch);
    for (int pass = 0; pass < 2; ++pass) {
        cudaError_t e = cudaMemsetAsync(W.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st);
        if (e != cudaSuccess) return e;
        if (pass == 0) k_gd_camera_base<<<(n_base + 255) / 256, 256, 0, st>>>(F, W, n_int, valid);
        else k_gd_camera_shift<<<(4 * n_base + 255) / 256, 256, 0, st>>>(F, W, n_int, valid);
        for (uint32_t d = 0; d < F.max_depth; ++d) {
            e = d == 0 && !count_stats ? pt_launch_extend_camera(S, W, num_sms, st)
                                       : pt_launch_extend(S, W, d, num_sms, st, 0u, count_stats);
            if (e != cudaSuccess) return e;
            if (pass == 0) k_gd_shade<false><<<num_sms * 8, 256, 0, st>>>(S, F, W, d, n_base, valid);
            else k_gd_shade<true><<<num_sms * 8, 256, 0, st>>>(S, F, W, d, n_base, valid);
            if ((e = pt_launch_connect(S, W, d, num_sms, st, count_stats)) != cudaSuccess) return e;
        }
        if (count_stats) k_ray_stats<<<1, 1, 0, st>>>(W, F.max_depth);
    }
    return cudaGetLastError();
}

cudaError_t gdpt_fold_frames(const PTFrame& F, const Workspace& W, float* const bufs[8], float* out, cudaStream_t st) {
    const uint32_t w = F.width, h = F.height;
    const uint32_t n_int = w >= 3 && h >= 3 ? (w - 2) * (h - 2) : 0u;
    // per frame, in order: its running means, then PBRendering::gradientdomain's
    // reconstruction of them (the output of the last frame is the call's)
    for (uint32_t fr = 0; fr < F.frames; ++fr) {
        if (n_int)
            k_gd_accumulate<<<(n_int + 255) / 256, 256, 0, st>>>(F, W, n_int, fr, bufs[2], bufs[3], bufs[4], bufs[5],
                                                                 bufs[6]);
        const cudaError_t e = launch_gdpt_reconstruct(w, h, bufs[2], bufs[3], bufs[4], bufs[5], bufs[6], bufs[0],
                                                      bufs[1], bufs[7], out, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_raytrace(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st) {
    k_raytrace<<<(F.n_paths + 127) / 128, 128, 0, st>>>(S, F, img, err);
    return cudaGetLastError();
}

}  // namespace cupbr_b200
