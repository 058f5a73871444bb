// RenderingMethod::VOLUME, GRADIENTDOMAIN and RAYTRACER.
//
// VOLUME (VolumeRenderer.cu:11-310) and the GDPT paths
// (GradientDomain.cu:110-246) carry per-path state that changes the traced
// geometry (a path inside a VOLUME object only sees that object) or links
// five paths per pixel (a shift path stops where the base path's vertex is
// invalid), so each is one thread per pixel over the shared traversal code;
// the GDPT reconstruction (init_kernel + 50 optimization passes,
// GradientDomain.cu:248-350, 379-401) ping-pongs between two buffers instead
// of copying temp back each pass.  Arithmetic follows dev_common.cuh's
// contract, operation order the reference's.
#include "methods.hpp"

#include "shading.cuh"
#include "trace.cuh"

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
    __device__ void flush(uint64_t* stats) const {
        if (!on || !stats) return;
        atomicAdd((unsigned long long*)&stats[STAT_EXT_NODES], (unsigned long long)ext.nodes);
        atomicAdd((unsigned long long*)&stats[STAT_EXT_TRIS], (unsigned long long)ext.tris);
        atomicAdd((unsigned long long*)&stats[STAT_SH_NODES], (unsigned long long)sh.nodes);
        atomicAdd((unsigned long long*)&stats[STAT_SH_TRIS], (unsigned long long)sh.tris);
        atomicAdd((unsigned long long*)&stats[STAT_EXT_RAYS], (unsigned long long)ext_rays);
        atomicAdd((unsigned long long*)&stats[STAT_SH_RAYS], (unsigned long long)sh_rays);
    }
};

__device__ __forceinline__ bool closest(const DeviceScene& S, f3 o, f3 d, Surf& h, bool& ovf, MCount& mc) {
    float t;
    int32_t prim;
    uint32_t key;
    trace_scene_rt(false, mc.on, S, nullptr, 0, o, d, 0.0f, t, prim, key, ovf, mc.ext);
    mc.ext_rays += mc.on ? 1u : 0u;
    h.t = t;
    if (prim == HIT_NONE) return false;
    h.P = o + t * d;
    hit_normal(S, prim, h.P, h.N, h.obj);
    return true;
}

__device__ __forceinline__ bool visible(const DeviceScene& S, float dist, f3 o, f3 d, bool& ovf, MCount& mc) {
    float t;
    int32_t prim;
    uint32_t key;
    mc.sh_rays += mc.on ? 1u : 0u;
    return !trace_scene_rt(true, mc.on, S, nullptr, 0, o, d, dist, t, prim, key, ovf, mc.sh);
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

__global__ void k_volume(DeviceScene S, PTFrame F, float* __restrict__ img, uint32_t* err, uint64_t* stats) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= F.n_paths) return;
    MCount mc;
    mc.on = stats != nullptr;
    const float INF = __int_as_float(0x7f800000);
    uint32_t seed = tea4(tid, F.frame_index);
    const uint32_t py = tid / F.width, px = tid - F.width * py;
    f3 o, d;
    camera_ray(F, px, py, true, seed, o, d);
    f3 rad = splat(0.0f), rw = splat(1.0f);
    const uint32_t L = S.n_lights, use_env = S.env_w > 0 ? 1u : 0u;
    const float nl = (float)(L + use_env);
    bool inside = false, ovf = false;
    int32_t obj_index = 0;
    f3 ray_start = splat(0.0f), out_dir = splat(0.0f);
    const f3 scene_ss = xyz(S.vol_sigma_s), scene_sa = xyz(S.vol_sigma_a);
    const float scene_g = S.vol_sigma_s.w;
    for (uint32_t depth = 0; depth < F.max_depth; ++depth) {
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
            hit = closest(S, o, d, g, ovf, mc);
        }
        const f3 inc = -1.0f * d;
        if (!hit) {
            if (use_env) rad += rw * env_lookup(S, d);
            break;
        }
        const MatView m = object_material(S, g.obj);
        f3 vss = scene_ss, vsa = scene_sa;
        float vg = scene_g;
        if (inside) {  // the medium of the object the path is inside
            const MatView im = object_material(S, obj_index);
            vss = im.sigma_s;
            vsa = im.sigma_a;
            vg = im.g;
        }
        // handleMediumInteraction (VolumeRenderer.cu:88-212)
        bool handled = false;
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
                        for (uint32_t i = 0; i < 3; ++i) pdf += comp(st, i) * expf(-1.0f * comp(st, i) * t);
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
                            // physical estimator: the scene medium's light term
                            // carries its phase value too (the reference leaves
                            // it out, VolumeRenderer.cu:180-186)
                            att = splat(hg_phase(vg, -dot(inc, ldir)));
                        }
                        const f3 sst = scene_sa + scene_ss;
                        if (visible(S, dist, so, normalize(ldir), ovf, mc))
                            rad += nl * vexp(-1.0f * sst * fminf(dist, 100000000.0f)) * att * lrad * rw;
                        const float4 shg = sample_hg(vg, -1.0f * inc, seed);
                        out_dir = xyz(shg);
                        ray_start = Pe;
                        next_valid = true;
                    } else {
                        rw = splat(0.0f);
                    }
                } else {
                    float pdf = 0.0f;
                    for (uint32_t i = 0; i < 3; ++i) pdf += expf(-comp(st, i) * g.t);
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
                    rw = splat(0.0f);  // directIlluminationVolumetric :31-35
                } else {
                    f3 ldir;
                    float dist;
                    const f3 lrad = sample_nee(S, m, seed, g.P, inc, g.N, ldir, dist);
                    if (visible(S, dist, g.P + 0.001f * ldir, normalize(ldir), ovf, mc))
                        rad += nl * fmaxf(0.0f, dot(g.N, ldir)) *
                               vexp(-1.0f * (vss + vsa) * fminf(dist, 100000000.0f)) * brdf(m, inc, ldir, g.N) * lrad *
                               rw;
                }
                const float4 s = sample_direction(m, seed, inc, g.N);  // :72-86
                const f3 dir = xyz(s);
                if (!(norm(dir) == 0.0f)) {
                    rw = rw * fabsf(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
                    out_dir = dir;
                    ray_start = g.P;
                    next_valid = true;
                }
            }
            if (F.use_rr) {
                const float alpha = clampf(fmaxf(rw.x, fmaxf(rw.y, rw.z)), 0.0f, 1.0f);
                if (rnd(seed) > alpha || feq0(alpha)) break;
                rw = rw / alpha;
            }
        }
        if (!next_valid) break;
        o = ray_start + 0.001f * out_dir;
        d = normalize(out_dir);
    }
    if (ovf) atomicAdd(err, 1u);
    mc.flush(stats);
    float* q = img + 3 * (size_t)tid;
    if (F.frame_index > 0) {
        const float a = 1.0f / ((float)F.frame_index + 1.0f);
        rad = (1.0f - a) * mk(q[0], q[1], q[2]) + a * rad;
    }
    q[0] = rad.x; q[1] = rad.y; q[2] = rad.z;
}

// collect_radiance (GradientDomain.cu:110-158); the base path (shift ==
// false) records its valid vertices in `valid`, shift paths read it.
__device__ f3 gd_collect(const DeviceScene& S, f3 o, f3 d, uint32_t seed, uint32_t max_depth, bool shift,
                         uint64_t& valid, bool& ovf, MCount& mc) {
    f3 rad = splat(0.0f), rw = splat(1.0f);
    const uint32_t L = S.n_lights, use_env = S.env_w > 0 ? 1u : 0u;
    const float nl = (float)(L + use_env);
    if (!shift) valid = 0;
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        if (shift && !((valid >> depth) & 1ull)) break;
        Surf g;
        if (!closest(S, o, d, g, ovf, mc)) {
            if (use_env) rad += rw * env_lookup(S, d);
            break;
        }
        if (!shift) valid |= 1ull << depth;
        const f3 inc = -1.0f * d;
        const MatView m = object_material(S, g.obj);
        rad += rw * m.albedo_e;
        if (m.type != 3 && dot(g.N, inc) <= 0.0f) {
            rw = splat(0.0f);
        } else {
            f3 ldir;
            float dist;
            const f3 lrad = sample_nee(S, m, seed, g.P, inc, g.N, ldir, dist);
            if (visible(S, dist, g.P + 0.001f * ldir, normalize(ldir), ovf, mc))
                rad += nl * fmaxf(0.0f, dot(g.N, ldir)) * brdf(m, inc, ldir, g.N) * lrad * rw;
        }
        const float4 s = sample_direction(m, seed, inc, g.N);
        const f3 dir = xyz(s);
        if (norm(dir) == 0.0f) break;
        rw = rw * fabsf(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
        if (shift && is_zero(rw)) break;  // a shift path's later contributions are all zero
        o = g.P + 0.01f * dir;
        d = normalize(dir);
    }
    return rad;
}

__global__ void k_gdpt(DeviceScene S, PTFrame F, float* __restrict__ base, float* __restrict__ gxf,
                       float* __restrict__ gxb, float* __restrict__ gyf, float* __restrict__ gyb, uint32_t* err,
                       uint64_t* stats) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= F.n_paths) return;
    const uint32_t py = tid / F.width, px = tid - F.width * py;
    if (px == 0 || px == F.width - 1 || py == 0 || py == F.height - 1) return;
    uint32_t seed = tea4(tid, F.frame_index);
    const int off[5][2] = {{0, 0}, {-1, 0}, {1, 0}, {0, 1}, {0, -1}};  // base, left, right, up, down
    f3 o[5], d[5];
    uint32_t seeds[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        camera_ray(F, (uint32_t)((int)px + off[k][0]), (uint32_t)((int)py + off[k][1]), true, seed, o[k], d[k]);
        seeds[k] = seed;
    }
    bool ovf = false;
    uint64_t valid = 0;
    MCount mc;
    mc.on = stats != nullptr;
    f3 Lr[5];
    Lr[0] = gd_collect(S, o[0], d[0], seeds[0], F.max_depth, false, valid, ovf, mc);
    for (int k = 1; k < 5; ++k) Lr[k] = gd_collect(S, o[k], d[k], seeds[k], F.max_depth, true, valid, ovf, mc);
    mc.flush(stats);
    f3 out[5] = {Lr[0], 0.5f * (Lr[0] - Lr[1]), 0.5f * (Lr[2] - Lr[0]), 0.5f * (Lr[0] - Lr[4]),
                 0.5f * (Lr[3] - Lr[0])};
    float* bufs[5] = {base, gxf, gxb, gyf, gyb};
    const float a = 1.0f / ((float)F.frame_index + 1.0f);
    for (int k = 0; k < 5; ++k) {
        float* q = bufs[k] + 3 * (size_t)tid;
        f3 v = out[k];
        if (F.frame_index > 0) v = (1.0f - a) * mk(q[0], q[1], q[2]) + a * v;
        q[0] = v.x; q[1] = v.y; q[2] = v.z;
    }
    if (ovf) atomicAdd(err, 1u);
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
// copy_border: the border pixels of dst take src's (see launch_gdpt).
__global__ void k_gdpt_opt(uint32_t w, uint32_t h, const float* __restrict__ src, const float* __restrict__ gx,
                           const float* __restrict__ gy, float* __restrict__ dst, int copy_border) {
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
__global__ void k_raytrace(DeviceScene S, PTFrame F, float* __restrict__ img, uint32_t* err) {
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

cudaError_t launch_volume(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st,
                          uint64_t* stats) {
    k_volume<<<(F.n_paths + 127) / 128, 128, 0, st>>>(S, F, img, err, stats);
    return cudaGetLastError();
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
    for (int i = 0; i < 50; ++i) {
        const float* src = (i & 1) ? temp : out;
        float* dst = (i & 1) ? out : temp;
        k_gdpt_opt<<<(n + 255) / 256, 256, 0, st>>>(w, h, src, gx, gy, dst, i & 1);
    }
    return cudaGetLastError();
}

cudaError_t launch_gdpt(const DeviceScene& S, const PTFrame& F, float* const bufs[8], float* out, uint32_t* err,
                        cudaStream_t st, uint64_t* stats) {
    // bufs: gx, gy, base, gxf, gxb, gyf, gyb, temp
    const uint32_t n = F.n_paths, w = F.width, h = F.height;
    k_gdpt<<<(n + 127) / 128, 128, 0, st>>>(S, F, bufs[2], bufs[3], bufs[4], bufs[5], bufs[6], err, stats);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_gdpt_reconstruct(w, h, bufs[2], bufs[3], bufs[4], bufs[5], bufs[6], bufs[0], bufs[1], bufs[7], out,
                                   st);
}

cudaError_t launch_raytrace(const DeviceScene& S, const PTFrame& F, float* img, uint32_t* err, cudaStream_t st) {
    k_raytrace<<<(F.n_paths + 127) / 128, 128, 0, st>>>(S, F, img, err);
    return cudaGetLastError();
}

}  // namespace cupbr_b200
