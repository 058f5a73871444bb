// Heterogeneous participating media: a density grid rendered by delta /
// weighted tracking with ratio-tracking transmittance, and its adjoint by
// path replay.  No counterpart in the reference (its VolumeRenderer.cu has a
// homogeneous medium only).
//
// Medium: density sigma(x) = grid[voxel(x)] (nearest voxel) inside the grid
// box, zero outside; sigma_s = albedo * sigma, Henyey-Greenstein phase (g);
// majorant sigma_bar >= every grid value.
//
// Free flight along a segment: tentative points at exponential steps of rate
// sigma_bar, clipped to the grid box and the closest surface.  At a point of
// density s:
//   analog delta tracking (q == 0): real with probability s / sigma_bar; the
//     real event scatters with weight albedo;
//   weighted tracking (0 < q < 1): if s > 0, real with the FIXED probability
//     q and weight albedo * s / (sigma_bar q); otherwise null with weight
//     (1 - s / sigma_bar) / (1 - q) (s == 0: null, weight 1).
// Weighted tracking is unbiased and, for fixed random numbers, a smooth
// function of every positive density -- the function the adjoint
// differentiates and central differences check.
// Shadow rays: ratio tracking, T = prod_k (1 - s_k / sigma_bar).
//
// Surfaces follow the path tracer (emission, one light sample, BSDF sample;
// back-facing hits end the path), with the light term attenuated by T.
// Scattering in the medium: one light sample weighted by the phase function
// and T, then a phase-function sample (weight 1).  Per vertex the random
// numbers are drawn as: free flight, light pick, light sample, ratio
// tracking, next direction.
//
// Wavefront, as the path tracer: per depth the persistent closest-hit
// kernel; k_medium_flight (free flight, persistent, sorting the paths into
// medium and surface vertices); k_medium_scatter and k_medium_surface (the
// vertices' light terms and next rays); k_medium_transmit (the light terms'
// ratio tracking, persistent); then the shadow rays -- the path tracer's
// k_connect when rendering the image, k_medium_connect in the gradient's two
// replays.
//
// Adjoint (path replay, no stored vertices): a forward wavefront gives every
// path's radiance L (summed in double); a second wavefront replays the same
// paths with the remaining radiance L_rem = L minus what has been emitted so
// far (taken out of the double sum), adding dot(dLoss/dI, L_rem) * dlog(w)/dtheta
// for every path weight w and dot(dLoss/dI, C) * dlog(C)/dtheta for every
// visible light term C:
//   null   : dlog/dsigma_v = -1 / (sigma_bar - sigma_v)
//   real   : dlog/dsigma_v = 1 / sigma_v,  dlog/dalbedo = 1 / albedo
//   ratio T: dlog/dsigma_v = -1 / (sigma_bar - sigma_v) per tracked point
//            (replayed from the saved RNG state once C is known visible)
//   Lambert: dlog/dalbedo_d[c] = 1 / albedo_d[c] (light term, and the sampled
//            weight -- applied at the next vertex, after that vertex's
//            light term has left L_rem)
//   light  : dlog C/dradiance[c] = 1 / radiance[c]
//   emission at a surface hit: dL/dalbedo_e[c] = beta[c] (the path weight
//            there), also for a surface that emits nothing yet
#include "medium.hpp"

#include <algorithm>

#include "shading.cuh"
#include "trace.cuh"
#include "wavefront.cuh"

namespace cupbr_b200 {

namespace {

// What a wavefront does with each path's radiance: RENDER sums it in float
// (the image); LSUM sums it in double (the L the adjoint replay starts
// from); ADJ replays the path taking every term out of that double sum, so
// L_rem = L - (terms so far) carries no float cancellation residue into
// the gradients of a path's last vertices.
enum WaveMode : int { RENDER = 0, LSUM = 1, ADJOINT = 2 };

// Frames [sample0, sample0 + frames) of one wavefront: path p is frame
// p / pixels of pixel p % pixels.
struct MediumBatch {
    uint32_t pixels, frames, n_paths, sample0;
};

__device__ __forceinline__ bool box_interval(const MediumGrid& G, f3 o, f3 d, float& ta, float& tb) {
    ta = 0.0f;
    tb = __int_as_float(0x7f800000);
    const float os[3] = {o.x, o.y, o.z}, ds[3] = {d.x, d.y, d.z};
    const float lo[3] = {G.lo.x, G.lo.y, G.lo.z}, hi[3] = {G.hi.x, G.hi.y, G.hi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (ds[a] == 0.0f) {
            if (os[a] < lo[a] || os[a] > hi[a]) return false;
            continue;
        }
        const float inv = 1.0f / ds[a];
        float t0 = (lo[a] - os[a]) * inv, t1 = (hi[a] - os[a]) * inv;
        if (t0 > t1) {
            const float tt = t0;
            t0 = t1;
            t1 = tt;
        }
        ta = t0 > ta ? t0 : ta;
        tb = t1 < tb ? t1 : tb;
    }
    return ta < tb;
}

__device__ __forceinline__ uint32_t voxel_of(const MediumGrid& G, f3 x) {
    int ix = (int)((x.x - G.lo.x) * G.inv_cell.x);
    int iy = (int)((x.y - G.lo.y) * G.inv_cell.y);
    int iz = (int)((x.z - G.lo.z) * G.inv_cell.z);
    ix = min(max(ix, 0), (int)G.nx - 1);
    iy = min(max(iy, 0), (int)G.ny - 1);
    iz = min(max(iz, 0), (int)G.nz - 1);
    return ((uint32_t)iz * G.ny + (uint32_t)iy) * G.nx + (uint32_t)ix;
}

__device__ __forceinline__ float free_step(const MediumGrid& G, uint32_t& seed) {
    return -logf(1.0f - rnd(seed)) * G.inv_majorant;
}

__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// A light term's ratio tracking draws from its own stream, seeded from the
// path's state right after the light sample (the path's stream goes on to
// the next direction), so it can run in a kernel of its own.
__host__ __device__ __forceinline__ uint32_t ratio_seed(uint32_t path_seed) { return tea4(path_seed, 1u); }

// Ratio-tracking transmittance of [0, len] along (o, d).  With g_grid the
// walk adds scale * dlogT/dsigma_v = -scale / (sigma_bar - sigma_v) per point.
__device__ __forceinline__ float ratio_track(const MediumGrid& G, f3 o, f3 d, float len, uint32_t& seed,
                                             float* g_grid, float scale, bool& ovf, uint32_t& lookups) {
    float ta, tb;
    if (!box_interval(G, o, d, ta, tb)) return 1.0f;
    tb = fminf(tb, len);
    float T = 1.0f, t = ta;
    for (int k = 0;; ++k) {
        if (k == MEDIUM_MAX_EVENTS) {
            ovf = true;
            break;
        }
        t += free_step(G, seed);
        if (!(t < tb)) break;
        const uint32_t v = voxel_of(G, o + t * d);
        const float s = __ldg(&G.density[v]);
        ++lookups;
        T *= 1.0f - s * G.inv_majorant;
        if (g_grid) atomicAdd(&g_grid[v], -scale / (G.majorant - s));
    }
    return T;
}

__device__ __forceinline__ void add_albedo_grad(float* ga, f3 delta, f3 v, f3 albedo) {
    if (albedo.x != 0.0f) atomicAdd(&ga[0], delta.x * v.x / albedo.x);
    if (albedo.y != 0.0f) atomicAdd(&ga[1], delta.y * v.y / albedo.y);
    if (albedo.z != 0.0f) atomicAdd(&ga[2], delta.z * v.z / albedo.z);
}

__device__ __forceinline__ f3 pixel_delta(const float* grad_img, uint32_t pixel, uint32_t spp) {
    const float* gi = grad_img + 3 * (size_t)pixel;
    return mk(gi[0], gi[1], gi[2]) / (float)spp;
}

__device__ __forceinline__ void lsum_add(double* l, uint32_t pid, f3 c, double sign) {
    double* q = l + 3 * (size_t)pid;
    q[0] += sign * (double)c.x;
    q[1] += sign * (double)c.y;
    q[2] += sign * (double)c.z;
}
__device__ __forceinline__ f3 lsum_get(const double* l, uint32_t pid) {
    const double* q = l + 3 * (size_t)pid;
    return mk((float)q[0], (float)q[1], (float)q[2]);
}

// Shared-memory copy of the parameter gradients (np_smem entries, 0 = use
// global memory directly).
__device__ __forceinline__ float* params_begin(float* s_params, uint32_t np_smem, float* g_params) {
    for (uint32_t k = threadIdx.x; k < np_smem; k += blockDim.x) s_params[k] = 0.0f;
    __syncthreads();
    return np_smem ? s_params : g_params;
}
__device__ __forceinline__ void params_end(const float* s_params, uint32_t np_smem, float* g_params) {
    if (!np_smem) return;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < np_smem; k += blockDim.x)
        if (s_params[k] != 0.0f) atomicAdd(&g_params[k], s_params[k]);
}

// TracingDetail.h:15-30 camera rays (as the path tracer's k_camera) into ray
// queue 0: (origin, path), (direction, seed), (1, pending Lambert object + 1
// = 0).  RENDER / LSUM clear the path's radiance sum; ADJOINT keeps it (it
// is the L_rem of the replay) and enqueues only paths whose pixel has a
// nonzero dLoss/dI.
template <int MODE>
__global__ void k_medium_camera(MediumParams P, MediumBatch B, Workspace W, double* __restrict__ lsum,
                                const float* __restrict__ grad_img) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    bool push = false;
    f3 o = P.cam_pos, d = mk(0.0f, 0.0f, 1.0f);
    uint32_t seed = 0;
    if (p < B.n_paths) {
        const uint32_t fr = p / B.pixels;
        const uint32_t tid = p - fr * B.pixels;
        seed = tea4(tid, B.sample0 + fr);
        const uint32_t py = tid / P.width, px = tid - P.width * py;
        const float jx = rnd(seed);
        const float jy = rnd(seed);
        const float rx = 2.0f * (((float)px + jx) / (float)P.width - 0.5f);
        const float ry = 2.0f * (((float)py + jy) / (float)P.height - 0.5f);
        const f3 wp = P.cam_pos + P.cam_z + rx * P.cam_x + ry * P.cam_y;
        d = normalize(wp - P.cam_pos);
        if (MODE == ADJOINT) {
            push = !is_zero(pixel_delta(grad_img, tid, P.spp));
        } else {
            push = true;
            if (MODE == RENDER) W.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            else lsum[3 * (size_t)p] = lsum[3 * (size_t)p + 1] = lsum[3 * (size_t)p + 2] = 0.0;
        }
    }
    const uint32_t slot = claim_slot(push, &W.ctr[CTR_RAYS + 0]);
    if (push) {
        float4* q = W.rays[0] + 3 * (size_t)slot;
        q[0] = f4(o, __uint_as_float(p));
        q[1] = f4(d, __uint_as_float(seed));
        q[2] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    }
}

// Free flight of every ray-queue entry through the grid up to its closest
// hit, sorting the paths into medium vertices (a real collision; front of
// `verts`) and surface vertices (back of `verts`): (position, path),
// (direction, RNG state), (weight, primitive ref for a surface).
// Persistent: a lane takes the next entry as soon as its flight ends (one
// atomicAdd per warp) and advances in rounds of FLIGHT_ROUND steps, so
// flights of different lengths keep a warp full.  The adjoint adds the
// pending Lambert weight gradient of the previous vertex and the free-flight
// gradients.
constexpr int FLIGHT_ROUND = 4;
constexpr int FLIGHT_BLOCKS_PER_SM = 4;

template <int MODE>
__global__ void __launch_bounds__(256) k_medium_flight(DeviceScene S, MediumGrid G, MediumParams P, MediumBatch B,
                                                       Workspace W, float4* __restrict__ verts, uint32_t capacity,
                                                       uint32_t depth, const double* __restrict__ lsum,
                                                       const float* __restrict__ grad_img, float* g_grid,
                                                       float* g_params, uint32_t np_smem, uint32_t* err,
                                                       unsigned long long* stats) {
    constexpr bool ADJ = MODE == ADJOINT;
    extern __shared__ float s_params[];
    float* gp = ADJ ? params_begin(s_params, np_smem, g_params) : nullptr;
    const uint32_t count = W.ctr[CTR_RAYS + depth];
    uint32_t* fetch = &W.ctr[CTR_FFETCH + depth];
    const float4* __restrict__ q = W.rays[depth & 1];
    const unsigned full = 0xffffffffu;
    const uint32_t lane = lane_id();
    bool have = false, exhausted = false, fin = false, scatter = false, ovf = false;
    uint32_t idx = 0, pid = 0, seed = 0, lookups = 0;
    int32_t prim = HIT_NONE;
    int steps = 0;
    f3 o = splat(0.0f), d = splat(0.0f), beta = splat(0.0f), x = splat(0.0f);
    f3 delta = splat(0.0f), Lrem = splat(0.0f);
    float t = 0.0f, tb = 0.0f, ts = 0.0f;
    float g_albedo = 0.0f;
    for (;;) {
        const bool want = !have && !exhausted;
        const unsigned m = __ballot_sync(full, want);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(fetch, (uint32_t)__popc(m));
            base = __shfl_sync(full, base, leader);
            if (want) {
                idx = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
                if (idx < count) {
                    const float4 q0 = __ldg(&q[3 * (size_t)idx]);
                    const float4 q1 = __ldg(&q[3 * (size_t)idx + 1]);
                    const float4 q2 = __ldg(&q[3 * (size_t)idx + 2]);
                    o = xyz(q0);
                    d = xyz(q1);
                    pid = __float_as_uint(q0.w);
                    seed = __float_as_uint(q1.w);
                    beta = xyz(q2);
                    const float2 h = W.hits[idx];
                    ts = h.x;
                    prim = __float_as_int(h.y);
                    if (ADJ) {
                        delta = pixel_delta(grad_img, pid % B.pixels, P.spp);
                        Lrem = lsum_get(lsum, pid);
                        const uint32_t pend = __float_as_uint(q2.w);
                        if (pend != 0u) {  // sampled Lambert weight of the previous vertex
                            const MatView pm =
                                load_material(S.materials, __float_as_int(__ldg(&S.objects[pend - 1u].hi).w));
                            add_albedo_grad(gp + 1 + 3 * (pend - 1u), delta, Lrem, pm.albedo_d);
                        }
                    }
                    scatter = false;
                    steps = 0;
                    float ta;
                    fin = !box_interval(G, o, d, ta, tb);  // no grid along the ray: no draws at all
                    if (!fin) {
                        tb = fminf(tb, ts);
                        t = ta;
                    }
                    have = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__ballot_sync(full, have)) break;
        if (have && !fin) {
            for (int r = 0; r < FLIGHT_ROUND; ++r) {
                if (steps++ == MEDIUM_MAX_EVENTS) {
                    ovf = true;
                    beta = splat(0.0f);
                    fin = true;
                    break;
                }
                t += free_step(G, seed);
                if (!(t < tb)) {
                    fin = true;
                    break;
                }
                const f3 xp = o + t * d;
                const uint32_t v = voxel_of(G, xp);
                const float s = __ldg(&G.density[v]);
                ++lookups;
                const float xi = rnd(seed);
                bool real;
                if (P.q <= 0.0f) {
                    real = xi < s * G.inv_majorant;
                    if (real) {
                        beta = P.albedo * beta;
                        if (ADJ) g_albedo += dot3(delta, Lrem) / P.albedo;
                    }
                } else {
                    real = s > 0.0f && xi < P.q;
                    if (real) {
                        beta = (P.albedo * s * G.inv_majorant * P.inv_q) * beta;
                        if (ADJ) {
                            const float lr = dot3(delta, Lrem);
                            atomicAdd(&g_grid[v], lr / s);
                            g_albedo += lr / P.albedo;
                        }
                    } else if (s > 0.0f) {
                        beta = ((1.0f - s * G.inv_majorant) * P.inv_one_minus_q) * beta;
                        if (ADJ) atomicAdd(&g_grid[v], -dot3(delta, Lrem) / (G.majorant - s));
                    }
                }
                if (real) {
                    scatter = true;
                    x = xp;
                    fin = true;
                    break;
                }
            }
        }
        const bool done = have && fin;
        const bool push_m = done && scatter && !is_zero(beta);
        const bool push_s = done && !scatter && prim != HIT_NONE && !is_zero(beta);
        const uint32_t ms = claim_slot(push_m, &W.ctr[CTR_MVERT + depth]);
        if (push_m) {
            float4* e = verts + 3 * (size_t)ms;
            e[0] = f4(x, __uint_as_float(pid));
            e[1] = f4(d, __uint_as_float(seed));
            e[2] = f4(beta, 0.0f);
        }
        const uint32_t ss = claim_slot(push_s, &W.ctr[CTR_SVERT + depth]);
        if (push_s) {
            float4* e = verts + 3 * (size_t)(capacity - 1u - ss);
            e[0] = f4(o + ts * d, __uint_as_float(pid));
            e[1] = f4(d, __uint_as_float(seed));
            e[2] = f4(beta, __int_as_float(prim));
        }
        if (done) have = false;
    }
    if (ovf) atomicAdd(err, 1u);
    if (stats) {
        unsigned long long n = lookups;
        for (int off = 16; off > 0; off >>= 1) n += __shfl_down_sync(full, n, off);
        if (lane == 0) atomicAdd(&stats[0], n);
    }
    if (ADJ) {
        for (int off = 16; off > 0; off >>= 1) g_albedo += __shfl_down_sync(full, g_albedo, off);
        if (lane == 0 && g_albedo != 0.0f) atomicAdd(&gp[0], g_albedo);
        params_end(s_params, np_smem, g_params);
    }
}

// Medium vertices: the light term (phase function; its ratio tracking runs
// later, in k_medium_transmit) and the phase-function sample of the next ray.
__global__ void __launch_bounds__(256) k_medium_scatter(DeviceScene S, MediumParams P, Workspace W,
                                                        const float4* __restrict__ verts,
                                                        float4* __restrict__ shadow_aux, uint32_t depth) {
    const uint32_t count = W.ctr[CTR_MVERT + depth];
    float4* __restrict__ qn = W.rays[(depth + 1) & 1];
    const bool last = depth + 1 >= P.max_depth;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nl = S.n_lights;
    for (uint32_t i0 = warp * 32u; i0 < count; i0 += nwarps * 32u) {
        const uint32_t i = i0 + lane_id();
        bool push_sh = false, push_ext = false;
        float4 sh0, sh1, sh2, shx, ex0, ex1, ex2;
        if (i < count) {
            const float4 v0 = __ldg(&verts[3 * (size_t)i]), v1 = __ldg(&verts[3 * (size_t)i + 1]);
            const float4 v2 = __ldg(&verts[3 * (size_t)i + 2]);
            const f3 x = xyz(v0), d = xyz(v1), beta = xyz(v2);
            const uint32_t pid = __float_as_uint(v0.w);
            uint32_t seed = __float_as_uint(v1.w);
            if (nl > 0) {
                const uint32_t li = (uint32_t)(rnd(seed) * (float)nl);
                f3 ldir;
                float dist;
                const f3 lrad = sample_light(S.lights, li, seed, x, ldir, dist);
                const f3 sd = normalize(ldir);
                const f3 C = ((float)nl * hg_phase(P.g, dot(d, sd))) * (lrad * beta);
                push_sh = !is_zero(C);  // a zero term changes neither L nor a gradient
                sh0 = f4(x, dist);
                sh1 = f4(sd, __uint_as_float(pid));
                sh2 = f4(C, 0.0f);
                shx = make_float4(__uint_as_float(ratio_seed(seed)), __uint_as_float(li), 0.0f, 0.0f);
            }
            const float4 sp = sample_hg(P.g, d, seed);
            if (!last) {
                push_ext = true;
                ex0 = f4(x, __uint_as_float(pid));
                ex1 = f4(normalize(xyz(sp)), __uint_as_float(seed));
                ex2 = f4(beta, 0.0f);
            }
        }
        const uint32_t ss = claim_slot(push_sh, &W.ctr[CTR_SHADOW + depth]);
        if (push_sh) {
            float4* e = W.shadow + 3 * (size_t)ss;
            e[0] = sh0;
            e[1] = sh1;
            e[2] = sh2;
            shadow_aux[ss] = shx;
        }
        const uint32_t es = claim_slot(push_ext, &W.ctr[CTR_RAYS + depth + 1]);
        if (push_ext) {
            float4* e = qn + 3 * (size_t)es;
            e[0] = ex0;
            e[1] = ex1;
            e[2] = ex2;
        }
    }
}

// Surface vertices: emission, the light term (ratio tracking later) and the
// BSDF sample of the next ray, as the path tracer; the adjoint adds the
// emission gradient and takes the emission out of L_rem.
template <int MODE>
__global__ void __launch_bounds__(256, 3) k_medium_surface(DeviceScene S, MediumParams P, MediumBatch B, Workspace W,
                                                          const float4* __restrict__ verts, uint32_t capacity,
                                                          float4* __restrict__ shadow_aux, uint32_t depth,
                                                          double* __restrict__ lsum,
                                                          const float* __restrict__ grad_img, float* g_params,
                                                          uint32_t np_smem) {
    constexpr bool ADJ = MODE == ADJOINT;
    extern __shared__ float s_params[];
    float* gp = ADJ ? params_begin(s_params, np_smem, g_params) : nullptr;
    const uint32_t count = W.ctr[CTR_SVERT + depth];
    float4* __restrict__ qn = W.rays[(depth + 1) & 1];
    const bool last = depth + 1 >= P.max_depth;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nl = S.n_lights;
    for (uint32_t i0 = warp * 32u; i0 < count; i0 += nwarps * 32u) {
        const uint32_t i = i0 + lane_id();
        bool push_sh = false, push_ext = false;
        float4 sh0, sh1, sh2, shx, ex0, ex1, ex2;
        if (i < count) {
            const float4* e = verts + 3 * (size_t)(capacity - 1u - i);
            const float4 v0 = __ldg(e), v1 = __ldg(e + 1), v2 = __ldg(e + 2);
            const f3 Pp = xyz(v0), d = xyz(v1);
            f3 beta = xyz(v2);
            const uint32_t pid = __float_as_uint(v0.w);
            uint32_t seed = __float_as_uint(v1.w);
            const int32_t prim = __float_as_int(v2.w);
            f3 N;
            int32_t obj;
            hit_normal(S, prim, Pp, N, obj);
            const MatView m = load_material(S.materials, __float_as_int(__ldg(&S.objects[obj].hi).w));
            const f3 inc = -1.0f * d;
            const f3 Ce = beta * m.albedo_e;
            if (ADJ) {
                const f3 delta = pixel_delta(grad_img, pid % B.pixels, P.spp);
                float* ge = gp + medium_emission_offset(S.n_objects) + 3 * obj;
                if (delta.x != 0.0f && beta.x != 0.0f) atomicAdd(&ge[0], delta.x * beta.x);
                if (delta.y != 0.0f && beta.y != 0.0f) atomicAdd(&ge[1], delta.y * beta.y);
                if (delta.z != 0.0f && beta.z != 0.0f) atomicAdd(&ge[2], delta.z * beta.z);
            }
            if (!is_zero(Ce)) {
                if (MODE == RENDER) {
                    const float4 r = W.radiance[pid];
                    W.radiance[pid] = make_float4(r.x + Ce.x, r.y + Ce.y, r.z + Ce.z, 0.0f);
                } else {
                    lsum_add(lsum, pid, Ce, ADJ ? -1.0 : 1.0);
                }
            }
            if (m.type == 3 || dot(N, inc) > 0.0f) {
                const uint32_t lam = m.type == 0 ? (uint32_t)obj + 1u : 0u;
                if (nl > 0) {
                    const uint32_t li = (uint32_t)(rnd(seed) * (float)nl);
                    f3 ldir;
                    float dist;
                    const f3 lrad = sample_light(S.lights, li, seed, Pp, ldir, dist);
                    const f3 so = Pp + 0.001f * ldir, sd = normalize(ldir);
                    const f3 C = ((float)nl * fmaxf(0.0f, dot(N, ldir))) * (brdf(m, inc, ldir, N) * lrad * beta);
                    push_sh = !is_zero(C);
                    sh0 = f4(so, dist);
                    sh1 = f4(sd, __uint_as_float(pid));
                    sh2 = f4(C, 0.0f);
                    shx = make_float4(__uint_as_float(ratio_seed(seed)), __uint_as_float(li), __uint_as_float(lam),
                                      0.0f);
                }
                const float4 sp = sample_direction(m, seed, inc, N);
                const f3 dir = xyz(sp);
                if (!(norm(dir) < CUPBR_EPS)) {
                    beta = beta * fabsf(dot(dir, N)) * brdf(m, inc, dir, N) / sp.w;
                    if (!last && !is_zero(beta)) {
                        push_ext = true;
                        ex0 = f4(Pp + 0.01f * dir, __uint_as_float(pid));
                        ex1 = f4(normalize(dir), __uint_as_float(seed));
                        ex2 = f4(beta, __uint_as_float(lam));
                    }
                }
            }
        }
        const uint32_t ss = claim_slot(push_sh, &W.ctr[CTR_SHADOW + depth]);
        if (push_sh) {
            float4* e = W.shadow + 3 * (size_t)ss;
            e[0] = sh0;
            e[1] = sh1;
            e[2] = sh2;
            shadow_aux[ss] = shx;
        }
        const uint32_t es = claim_slot(push_ext, &W.ctr[CTR_RAYS + depth + 1]);
        if (push_ext) {
            float4* e = qn + 3 * (size_t)es;
            e[0] = ex0;
            e[1] = ex1;
            e[2] = ex2;
        }
    }
    if (ADJ) params_end(s_params, np_smem, g_params);
}

// Ratio-tracked transmittance of the depth's shadow rays, multiplied into
// their light terms (C = T * C).  Persistent: a lane takes the next shadow
// ray as soon as its own is done (one atomicAdd per warp for all lanes that
// need one) and every lane advances in rounds of TRANSMIT_ROUND steps, so a
// warp stays full although the rays' step counts differ.
constexpr int TRANSMIT_ROUND = 8;
constexpr int TRANSMIT_BLOCKS_PER_SM = 6;

__global__ void __launch_bounds__(256) k_medium_transmit(MediumGrid G, Workspace W,
                                                         const float4* __restrict__ shadow_aux, uint32_t depth,
                                                         uint32_t* err, unsigned long long* stats) {
    const uint32_t count = W.ctr[CTR_SHADOW + depth];
    uint32_t* fetch = &W.ctr[CTR_TFETCH + depth];
    const unsigned full = 0xffffffffu;
    const uint32_t lane = lane_id();
    bool have = false, exhausted = false, ovf = false;
    uint32_t idx = 0, seed = 0, lookups = 0;
    int steps = 0;
    f3 o = splat(0.0f), d = splat(0.0f);
    float t = 0.0f, tb = 0.0f, T = 1.0f;
    for (;;) {
        const bool want = !have && !exhausted;
        const unsigned m = __ballot_sync(full, want);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(fetch, (uint32_t)__popc(m));
            base = __shfl_sync(full, base, leader);
            if (want) {
                idx = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
                if (idx < count) {
                    const float4 e0 = W.shadow[3 * (size_t)idx], e1 = W.shadow[3 * (size_t)idx + 1];
                    o = xyz(e0);
                    d = xyz(e1);
                    seed = __float_as_uint(__ldg(&shadow_aux[idx]).x);
                    T = 1.0f;
                    steps = 0;
                    float ta;
                    if (box_interval(G, o, d, ta, tb)) {
                        tb = fminf(tb, e0.w);
                        t = ta;
                    } else {
                        t = 0.0f;  // outside the grid: the first step ends the walk with T = 1
                        tb = 0.0f;
                    }
                    have = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__ballot_sync(full, have)) break;
        if (have) {
            // A ratio-tracking point's position depends on the random step
            // lengths only, never on a density, so the round's density loads
            // are all issued before the first of them is used.
            float sk[TRANSMIT_ROUND];
            bool in[TRANSMIT_ROUND];
            bool done = false, over = false;
#pragma unroll
            for (int r = 0; r < TRANSMIT_ROUND; ++r) {
                in[r] = false;
                sk[r] = 0.0f;
                if (done) continue;
                if (steps++ == MEDIUM_MAX_EVENTS) {
                    over = done = true;
                    continue;
                }
                t += free_step(G, seed);
                if (!(t < tb)) {
                    done = true;
                    continue;
                }
                in[r] = true;
                sk[r] = __ldg(&G.density[voxel_of(G, o + t * d)]);
            }
#pragma unroll
            for (int r = 0; r < TRANSMIT_ROUND; ++r) {
                if (!in[r]) continue;
                T *= 1.0f - sk[r] * G.inv_majorant;
                ++lookups;
            }
            if (over) {
                ovf = true;
                T = 0.0f;
            }
            if (done) {
                float4* e = W.shadow + 3 * (size_t)idx + 2;
                const float4 c = *e;
                *e = make_float4(T * c.x, T * c.y, T * c.z, 0.0f);
                have = false;
            }
        }
    }
    if (ovf) atomicAdd(err, 1u);
    if (stats) {
        unsigned long long n = lookups;
        for (int off = 16; off > 0; off >>= 1) n += __shfl_down_sync(full, n, off);
        if (lane == 0) atomicAdd(&stats[1], n);
    }
}

// Shadow rays of the gradient pipeline.  LSUM: visible light terms join
// the path's double radiance sum.  ADJOINT: for every visible shadow ray,
// replay its ratio tracking for the density gradient, add the light (and
// Lambert albedo) gradients, and take the term out of the path's remaining
// radiance.
template <int MODE>
__global__ void __launch_bounds__(PT_TRACE_THREADS) k_medium_connect(DeviceScene S, MediumGrid G, MediumParams P,
                                                                     MediumBatch B, Workspace W,
                                                                     const float4* __restrict__ shadow_aux,
                                                                     uint32_t depth, double* __restrict__ lsum,
                                                                     const float* __restrict__ grad_img,
                                                                     float* g_grid, float* g_params, uint32_t np_smem,
                                                                     uint32_t* err) {
    extern __shared__ float4 s_dyn[];
    const uint32_t nsm = min(S.n_nodes, W.smem_nodes);
    float* s_params = reinterpret_cast<float*>(s_dyn + BVH_NODE_F4 * nsm);
    float* gp = params_begin(s_params, np_smem, g_params);
    bool ovf = false;
    persistent_trace<true, false>(
        S, W.shadow, 3, W.ctr[CTR_SHADOW + depth], &W.ctr[CTR_CFETCH + depth], W.smem_nodes, s_dyn,
        &W.err[ERR_STACK], W.stats, [&](uint32_t idx, const TravState& s) {
            if (s.hit) return;
            const float4* e = W.shadow + 3 * (size_t)idx;
            const float4 e0 = __ldg(e), e1 = __ldg(e + 1), e2 = __ldg(e + 2);
            const uint32_t pid = __float_as_uint(e1.w);
            const f3 C = xyz(e2);
            if (MODE == LSUM) {
                lsum_add(lsum, pid, C, 1.0);
                return;
            }
            const float4 ax = __ldg(&shadow_aux[idx]);
            const f3 delta = pixel_delta(grad_img, pid % B.pixels, P.spp);
            uint32_t seed_ratio = __float_as_uint(ax.x);
            uint32_t replayed = 0;
            ratio_track(G, xyz(e0), xyz(e1), e0.w, seed_ratio, g_grid, dot3(delta, C), ovf, replayed);
            const uint32_t li = __float_as_uint(ax.y), lam = __float_as_uint(ax.z);
            const f3 R = __ldg(&S.lights[li].pos).w == 0.0f ? xyz(__ldg(&S.lights[li].I))
                                                             : xyz(__ldg(&S.lights[li].L));
            add_albedo_grad(gp + medium_light_offset(S.n_objects) + 3 * li, delta, C, R);
            if (lam != 0u) {
                const MatView m = load_material(S.materials, __float_as_int(__ldg(&S.objects[lam - 1u].hi).w));
                add_albedo_grad(gp + 1 + 3 * (lam - 1u), delta, C, m.albedo_d);
            }
            lsum_add(lsum, pid, C, -1.0);
        });
    if (ovf) atomicAdd(err, 1u);
    params_end(s_params, np_smem, g_params);
}

// Queue sizes of an instrumented wavefront into stats[2..4].
__global__ void k_medium_count(Workspace W, uint32_t max_depth, uint32_t n_paths, unsigned long long* stats) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long rays = 0, shadow = 0;
    for (uint32_t d = 0; d < max_depth; ++d) {
        rays += W.ctr[CTR_RAYS + d];
        shadow += W.ctr[CTR_SHADOW + d];
    }
    stats[2] += rays;
    stats[3] += shadow;
    stats[4] += n_paths;
}

// Sums the wavefront's frames into img in frame order; the first batch
// starts from zero, the last divides by spp (mean = sum / spp).
__global__ void k_medium_accumulate(MediumParams P, MediumBatch B, Workspace W, float* __restrict__ img, bool first,
                                    bool final_batch) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= B.pixels) return;
    float* o = img + 3 * (size_t)tid;
    f3 acc = first ? splat(0.0f) : mk(o[0], o[1], o[2]);
    for (uint32_t fr = 0; fr < B.frames; ++fr) acc += xyz(W.radiance[(size_t)fr * B.pixels + tid]);
    if (final_batch) acc = acc / (float)P.spp;
    o[0] = acc.x;
    o[1] = acc.y;
    o[2] = acc.z;
}

uint32_t frames_per_batch(const MediumParams& P, const MediumWorkspace& W) {
    const uint32_t pixels = P.width * P.height;
    return std::max(1u, std::min(P.spp, W.capacity / pixels));
}

void no_mark() {}

// One wavefront over frames [B.sample0, B.sample0 + B.frames): RENDER and
// LSUM replay the paths forward, ADJOINT accumulates the gradients; mark()
// records the next profiling event (if any).
template <int MODE, typename Mark>
cudaError_t wavefront(const DeviceScene& S, const MediumGrid& G, const MediumParams& P, const MediumBatch& B,
                      const MediumWorkspace& W, const float* grad_img, float* g_grid, float* g_params, uint32_t* err,
                      int num_sms, cudaStream_t st, Mark mark) {
    const uint32_t np = medium_param_count(S.n_objects, S.n_lights);
    const uint32_t np_smem = MODE == ADJOINT && np <= MEDIUM_SMEM_PARAMS ? np : 0;
    const int connect_smem = (int)(std::min(S.n_nodes, W.pt.smem_nodes) * BVH_NODE_BYTES + np_smem * sizeof(float));
    unsigned long long* stats = MODE == RENDER ? W.stats : nullptr;
    cudaError_t e = cudaMemsetAsync(W.pt.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st);
    if (e != cudaSuccess) return e;
    mark();
    k_medium_camera<MODE><<<(B.n_paths + 255) / 256, 256, 0, st>>>(P, B, W.pt, W.lsum, grad_img);
    mark();
    for (uint32_t d = 0; d < P.max_depth; ++d) {
        if ((e = pt_launch_extend(S, W.pt, d, num_sms, st)) != cudaSuccess) return e;
        mark();
        k_medium_flight<MODE><<<num_sms * FLIGHT_BLOCKS_PER_SM, 256, np_smem * sizeof(float), st>>>(
            S, G, P, B, W.pt, W.verts, W.capacity, d, W.lsum, grad_img, g_grid, g_params, np_smem, err, stats);
        k_medium_scatter<<<num_sms * 8, 256, 0, st>>>(S, P, W.pt, W.verts, W.shadow_aux, d);
        k_medium_surface<MODE><<<num_sms * 8, 256, np_smem * sizeof(float), st>>>(
            S, P, B, W.pt, W.verts, W.capacity, W.shadow_aux, d, W.lsum, grad_img, g_params, np_smem);
        mark();
        k_medium_transmit<<<num_sms * TRANSMIT_BLOCKS_PER_SM, 256, 0, st>>>(G, W.pt, W.shadow_aux, d, err, stats);
        mark();
        if constexpr (MODE == RENDER) {
            if ((e = pt_launch_connect(S, W.pt, d, num_sms, st)) != cudaSuccess) return e;
        } else {
            k_medium_connect<MODE><<<num_sms * W.pt.trace_blocks_per_sm, PT_TRACE_THREADS, connect_smem, st>>>(
                S, G, P, B, W.pt, W.shadow_aux, d, W.lsum, grad_img, g_grid, g_params, np_smem, err);
        }
        mark();
    }
    return cudaGetLastError();
}

MediumBatch batch_at(const MediumParams& P, uint32_t s0, uint32_t fpb) {
    MediumBatch B;
    B.pixels = P.width * P.height;
    B.frames = std::min(fpb, P.spp - s0);
    B.n_paths = B.frames * B.pixels;
    B.sample0 = P.frame0 + s0;
    return B;
}

}  // namespace

uint32_t medium_batches(const MediumParams& P, const MediumWorkspace& W) {
    if (P.width * P.height == 0 || P.spp == 0) return 0;
    const uint32_t fpb = frames_per_batch(P, W);
    return (P.spp + fpb - 1) / fpb;
}

cudaError_t medium_render(const DeviceScene& S, const MediumGrid& G, const MediumParams& P, const MediumWorkspace& W,
                          float* img, uint32_t* err, int num_sms, cudaStream_t st, cudaEvent_t* ev) {
    const uint32_t pixels = P.width * P.height;
    if (pixels == 0 || P.spp == 0) return cudaSuccess;
    const uint32_t fpb = frames_per_batch(P, W);
    uint32_t ei = 0;
    auto mark = [&]() {
        if (ev) cudaEventRecord(ev[ei++], st);
    };
    for (uint32_t s0 = 0; s0 < P.spp; s0 += fpb) {
        const MediumBatch B = batch_at(P, s0, fpb);
        cudaError_t e = wavefront<RENDER>(S, G, P, B, W, nullptr, nullptr, nullptr, err, num_sms, st, mark);
        if (e != cudaSuccess) return e;
        if (W.stats) k_medium_count<<<1, 32, 0, st>>>(W.pt, P.max_depth, B.n_paths, W.stats);
        k_medium_accumulate<<<(pixels + 255) / 256, 256, 0, st>>>(P, B, W.pt, img, s0 == 0, s0 + B.frames >= P.spp);
        mark();
    }
    return cudaGetLastError();
}

cudaError_t medium_gradient(const DeviceScene& S, const MediumGrid& G, const MediumParams& P, const MediumWorkspace& W,
                            const float* grad_img, float* g_grid, float* g_params, uint32_t* err, int num_sms,
                            cudaStream_t st) {
    if (P.width * P.height == 0 || P.spp == 0) return cudaSuccess;
    const uint32_t fpb = frames_per_batch(P, W);
    for (uint32_t s0 = 0; s0 < P.spp; s0 += fpb) {
        const MediumBatch B = batch_at(P, s0, fpb);
        // replay 1: every path's radiance L (double sums)
        cudaError_t e = wavefront<LSUM>(S, G, P, B, W, grad_img, g_grid, g_params, err, num_sms, st, no_mark);
        if (e != cudaSuccess) return e;
        // replay 2: the same paths, accumulating the gradients
        e = wavefront<ADJOINT>(S, G, P, B, W, grad_img, g_grid, g_params, err, num_sms, st, no_mark);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

}  // namespace cupbr_b200
