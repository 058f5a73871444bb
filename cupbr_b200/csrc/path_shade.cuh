// Shading of one path vertex, shared by the wavefront shading stage, the
// per-path tail kernel (pathtracer.cu) and the persistent batch kernel
// (batch.cu).
#pragma once

#include "cache.hpp"
#include "pathtracer.hpp"
#include "shading.cuh"
#include "wavefront.cuh"

namespace cupbr_b200 {

// What shading one ray produced: a shadow-queue entry, the next ray, a
// cache query (cached frames).
struct ShadeOut {
    bool sh, ext, q;
    int32_t texel;       // albedo texel of the vertex (textured Lambert objects), else -1
    float4 s0, s1, s2;   // (origin, light distance), (direction, path), (contribution, -)
    float4 e0, e1, e2;   // (origin, path), (direction, seed), (throughput, -)
    float4 cq[RC_REC];
};

// One ray of ray queue[depth] with its hit h (PathTracer.cu:20-95 for one
// bounce): emission and env terms into the path radiance, light or env
// selection, NEE shadow ray, RR, BSDF sample.  CACHE: radiance-cache frames
// (CacheFrame): a path that is not a training path ends at its first
// front-facing hit at depth >= C.cache_depth that is not a mirror or glass
// (with C.specular, beyond the first cached depth, any material) with a cache
// query (the cache answers that vertex's emission, direct and indirect
// light); training paths record every vertex with the throughput that
// reached it and the radiance gathered before it, and are traced in full or,
// with C.train_end, end in a cache query at their first such hit at depth >=
// C.train_end.
// PHYS (CUPBR_ESTIMATOR_PHYSICAL, path tracer only): the environment's light
// term samples the environment map and both it and an escaping path's
// environment radiance are weighted by the power heuristic against the other
// technique; q2.w carries the density per solid angle with which the
// previous vertex's BSDF sampled this ray (0 for camera rays and delta
// lobes, whose escaping radiance counts in full).
// shade_core takes the path's radiance in `rad` (updated in place);
// shade_one keeps it in the workspace's per-path radiance.
template <bool CACHE, bool PHYS>
__device__ __forceinline__ void shade_core(const DeviceScene& S, const PTFrame& F, const CacheFrame& C, uint32_t depth,
                                           const float4& q0, const float4& q1, const float4& q2, float2 h, f3& rad,
                                           ShadeOut& so) {
    const bool last = depth + 1 >= F.max_depth;
    const uint32_t L = S.n_lights;
    const uint32_t use_env = S.env_w > 0 ? 1u : 0u;
    const uint32_t nl = L + use_env;
    const float INF = __int_as_float(0x7f800000);
    so.sh = so.ext = so.q = false;
    so.texel = -1;
    const f3 o = xyz(q0), d = xyz(q1);
    const uint32_t pid = __float_as_uint(q0.w);
    uint32_t seed = __float_as_uint(q1.w);
    f3 tp = xyz(q2);
    const int32_t prim = __float_as_int(h.y);
    if (prim == HIT_NONE) {
        if (use_env) {  // PathTracer.cu:127-135
            if (PHYS && q2.w > 0.0f) {
                float pe;
                const f3 le = env_lookup_pdf(S, d, pe);
                rad += tp * (le * mis_power(q2.w, pe / (float)nl));
            } else {
                rad += tp * env_lookup(S, d);
            }
        }
    } else {
        const float t = h.x;
        const f3 P = o + t * d;
        f3 N;
        int32_t obj;
        const uint32_t slot = prim_slot(prim);
        switch (prim_type(prim)) {
            case 0:
                N = xyz(__ldg(&S.tri_n[slot]));
                obj = __float_as_int(__ldg(&S.tris[3 * (size_t)slot + 1]).w);
                break;
            case 1: {
                float4 s0 = __ldg(&S.spheres[2 * (size_t)slot]);
                N = normalize(P - xyz(s0));
                obj = __float_as_int(__ldg(&S.spheres[2 * (size_t)slot + 1]).z);
                break;
            }
            case 2:
                N = xyz(__ldg(&S.quads[4 * (size_t)slot + 1]));
                obj = __ldg(&S.quad_obj[slot]);
                break;
            default: {
                float4 p1 = __ldg(&S.planes[2 * (size_t)slot + 1]);
                N = xyz(p1);
                obj = __float_as_int(p1.w);
                break;
            }
        }
        const int mat_idx = __float_as_int(__ldg(&S.objects[obj].hi).w);
        MatView m = load_material(S.materials, mat_idx);
        if (m.type == 0) {  // textured Lambert: the texel is the diffuse albedo
            f3 a;
            so.texel = tex_lookup(S, obj, P, a);
            if (so.texel >= 0) {
                m.albedo_d = a;
                m.albedo_d_over_pi = a / (float)3.14159265358979323846;
            }
        }
        const f3 inc = -1.0f * d;
        const bool facing = m.type == 3 || dot(N, inc) > 0.0f;
        if (CACHE) {
            const bool delta = m.type == 2 || m.type == 3;
            const bool cacheable = facing && (!delta || (C.specular && depth > C.cache_depth));
            so.cq[0] = f4(P, __uint_as_float(pid));
            so.cq[1] = f4(inc, m.roughness);
            so.cq[2] = f4(N, rad.x);
            so.cq[3] = f4(m.albedo_d, rad.y);
            so.cq[4] = f4(tp, rad.z);
            const bool train = C.train_stride != 0 && pid % C.train_stride == C.train_phase;
            if (train && cacheable && C.train_end != 0 && depth >= C.train_end) {
                // short training path: the cache supplies its tail
                so.q = true;
            } else if (train) {
                // training vertex: w of [0] flags a vertex the cache may answer,
                // w of [2..4] is the radiance gathered before it
                const uint32_t tidx = pid / C.train_stride;
                float4* v = C.tverts + RC_REC * ((size_t)tidx * F.max_depth + depth);
                v[0] = f4(P, cacheable ? 1.0f : 0.0f);
#pragma unroll
                for (int k = 1; k < (int)RC_REC; ++k) v[k] = so.cq[k];
                C.tcount[tidx] = depth + 1;
            } else if (cacheable && depth >= C.cache_depth) {
                so.q = true;
            }
            if (so.q) {
                so.cq[2].w = (float)(F.max_depth - depth);  // bounces left
                so.cq[3].w = 0.0f;
                so.cq[4].w = 0.0f;
            }
        }
        if (!so.q) rad += tp * m.albedo_e;  // PathTracer.cu:20-26
        if (so.q) {
            // the cache answers this vertex
        } else if (!facing) {
            // back-facing: throughput 0 (PathTracer.cu:37-41), path ends
        } else {
            // directIllumination, PathTracer.cu:43-72
            uint32_t ls = (uint32_t)(rnd(seed) * (float)nl);
            f3 ldir, lrad;
            float dist;
            if (ls != L) {
                lrad = sample_light(S.lights, ls, seed, P, ldir, dist);
            } else if (PHYS) {
                // environment by importance sampling; none at delta lobes
                dist = INF;
                ldir = N;
                lrad = splat(0.0f);
                if (use_env && !has_delta_lobe(m.type)) {
                    ldir = env_sample(S, seed);
                    float pe;
                    const f3 le = env_lookup_pdf(S, ldir, pe);
                    if (pe > 0.0f) lrad = le * (mis_power(pe / (float)nl, bsdf_pdf(m, inc, ldir, N)) / pe);
                }
            } else {
                float4 s = sample_direction(m, seed, inc, N);
                ldir = xyz(s);
                dist = INF;
                lrad = use_env ? env_lookup(S, ldir) / s.w : splat(0.0f);
            }
            f3 contrib = (float)nl * fmaxf(0.0f, dot(N, ldir)) * brdf(m, inc, ldir, N) * lrad * tp;
            if (!is_zero(contrib)) {
                so.sh = true;
                so.s0 = f4(P + 0.001f * ldir, dist);
                so.s1 = f4(normalize(ldir), __uint_as_float(pid));
                so.s2 = f4(contrib, 0.0f);
            }
            bool alive = true;
            if (F.use_rr) {  // PathTracer.cu:142-152
                float alpha = clampf(fmaxf(tp.x, fmaxf(tp.y, tp.z)), 0.0f, 1.0f);
                if (rnd(seed) > alpha || feq0(alpha)) alive = false;
                else tp = tp / alpha;
            }
            if (alive) {  // indirectIllumination, PathTracer.cu:76-95
                float4 s = sample_direction(m, seed, inc, N);
                f3 dir = xyz(s);
                if (!(norm(dir) < CUPBR_EPS)) {
                    tp = tp * fabsf(dot(dir, N)) * brdf(m, inc, dir, N) / s.w;
                    if (!last && !is_zero(tp)) {
                        so.ext = true;
                        so.e0 = f4(P + 0.01f * dir, __uint_as_float(pid));
                        so.e1 = f4(normalize(dir), __uint_as_float(seed));
                        so.e2 = f4(tp, PHYS && !has_delta_lobe(m.type) ? s.w : 0.0f);
                    }
                }
            }
        }
    }
}

// Material class of a hit for ordering the shading work: 0 miss, 1 diffuse
// (Lambert, Phong, volume interface), 2 GGX, 3 mirror or glass.
__device__ __forceinline__ uint32_t shade_class(const DeviceScene& S, float2 h) {
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
    const int mat_idx = __float_as_int(__ldg(&S.objects[obj].hi).w);
    const int type = (int)__ldg(&S.materials[mat_idx].e).w;
    return type == 4 ? 2u : (type == 2 || type == 3) ? 3u : 1u;
}

template <bool CACHE, bool PHYS, bool NC = true>
__device__ __forceinline__ void shade_one(const DeviceScene& S, const PTFrame& F, const Workspace& W,
                                          const CacheFrame& C, uint32_t depth, const float4& q0, const float4& q1,
                                          const float4& q2, float2 h, ShadeOut& so) {
    const uint32_t pid = __float_as_uint(q0.w);
    f3 rad = xyz(NC ? W.radiance[pid] : __ldcg(&W.radiance[pid]));
    shade_core<CACHE, PHYS>(S, F, C, depth, q0, q1, q2, h, rad, so);
    W.radiance[pid] = f4(rad, 0.0f);
}

// The shading stage of one depth over ray queue[depth] with blocks of 256
// threads striding over 256-ray chunks (k_shade, and the persistent batch
// kernel's shading stage): each chunk is shaded in material-class order
// (misses, diffuse, GGX, delta), so most warps run one BSDF.  A queue below
// C.tail_threshold is left to k_tail.
template <bool CACHE, bool PHYS, bool NC = true>
__device__ __forceinline__ void shade_stage(const DeviceScene& S, const PTFrame& F, const Workspace& W, uint32_t depth,
                                            const CacheFrame& C) {
    const uint32_t count = NC ? W.ctr[CTR_RAYS + depth] : __ldcg(&W.ctr[CTR_RAYS + depth]);
    if (count < C.tail_threshold) return;
    const float4* __restrict__ q = W.rays[depth & 1];
    float4* __restrict__ qn = W.rays[(depth + 1) & 1];
    // each chunk of 256 rays is shaded in material-class order (misses,
    // diffuse, GGX, delta), so most warps run one BSDF's code
    __shared__ uint32_t s_cnt[8][4];
    __shared__ uint32_t s_idx[256];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;

    for (uint32_t c0 = blockIdx.x * 256u; c0 < count; c0 += gridDim.x * 256u) {
        const uint32_t mine = c0 + threadIdx.x;
        uint32_t cls = 4;  // past the end
        if (mine < count) cls = shade_class(S, NC ? W.hits[mine] : __ldcg(&W.hits[mine]));
        uint32_t rank = 0;
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const unsigned m = __ballot_sync(full, cls == k);
            if (cls == k) rank = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) s_cnt[wid][k] = __popc(m);
        }
        __syncthreads();
        if (cls < 4) {
            uint32_t base = 0;
            for (uint32_t k = 0; k < cls; ++k)
                for (uint32_t w = 0; w < 8; ++w) base += s_cnt[w][k];
            for (uint32_t w = 0; w < wid; ++w) base += s_cnt[w][cls];
            s_idx[base + rank] = mine;
        }
        __syncthreads();
        const uint32_t i = threadIdx.x < count - c0 ? s_idx[threadIdx.x] : 0xFFFFFFFFu;
        ShadeOut so;
        so.sh = so.ext = so.q = false;
        if (i < count) {
            const float4 q0 = qload<NC>(&q[3 * (size_t)i]);
            const float4 q1 = qload<NC>(&q[3 * (size_t)i + 1]);
            const float4 q2 = qload<NC>(&q[3 * (size_t)i + 2]);
            shade_one<CACHE, PHYS, NC>(S, F, W, C, depth, q0, q1, q2, NC ? W.hits[i] : __ldcg(&W.hits[i]), so);
        }
        uint32_t ss = claim_slot(so.sh, &W.ctr[CTR_SHADOW + depth]);
        if (so.sh) {
            float4* e = W.shadow + 3 * (size_t)ss;
            e[0] = so.s0; e[1] = so.s1; e[2] = so.s2;
        }
        uint32_t es = claim_slot(so.ext, &W.ctr[CTR_RAYS + depth + 1]);
        if (so.ext) {
            float4* e = qn + 3 * (size_t)es;
            e[0] = so.e0; e[1] = so.e1; e[2] = so.e2;
        }
        if (CACHE) {
            uint32_t qs = claim_slot(so.q, C.n_queries);
            if (so.q) {
#pragma unroll
                for (int k = 0; k < (int)RC_REC; ++k) C.queries[(size_t)k * C.query_stride + qs] = so.cq[k];
            }
        }
        __syncthreads();  // s_cnt / s_idx of the next chunk
    }
}


}  // namespace cupbr_b200
