// Ray-primitive tests and BVH traversal (closest hit and any hit).
//
// Primitive tests repeat the reference's arithmetic in its order
// (TriangleDetail.h:21-57, SphereDetail.h:33-74, QuadDetail.h:21-57,
// PlaneDetail.h:19-46) so that the hit distance of every candidate equals the
// reference's.  Which candidate wins also follows the reference: a hit on an
// object with a finite box only counts if the reference's own slab test
// (AABBDetail.h:18-50, with its +EPSILON direction perturbation) accepts
// that box, and exact ties go to the smaller primitive key, where keys run
// in the leaf order of the reference's object BVH (first object in its
// depth-first order, then triangle index, MeshDetail.h:28-35).
//
// The SAH BVH itself is traversed with conservative FMA slab tests against
// boxes that the builder inflated, a per-thread short stack of (node, t_near)
// entries and near-child-first ordering.
#pragma once

#include "bvh_build.hpp"
#include "dev_common.cuh"

namespace cupbr_b200 {

#ifndef CUPBR_STACK_SIZE
#define CUPBR_STACK_SIZE 64
#endif

// TriangleDetail.h:21-57
__device__ __forceinline__ bool isect_tri(float4 a, float4 b, float4 c, f3 o, f3 d, float& t) {
    f3 v0v1 = xyz(b), v0v2 = xyz(c);
    f3 pvec = cross(d, v0v2);
    float det = dot(v0v1, pvec);
    if (feq0(det)) return false;
    float invDet = 1.0f / det;
    f3 tvec = o - xyz(a);
    float u = dot(tvec, pvec) * invDet;
    if (u < 0.0f || u > 1.0f) return false;
    f3 qvec = cross(tvec, v0v1);
    float v = dot(d, qvec) * invDet;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(v0v2, qvec) * invDet;
    return !(t < 0.0f);
}

// SphereDetail.h:33-74
__device__ __forceinline__ bool isect_sphere(float4 s0, float4 s1, f3 o, f3 d, float& t) {
    f3 OS = o - xyz(s0);
    float b = 2.0f * dot(d, OS);
    float c = dot(OS, OS) - s1.y;
    float disc = b * b - 4.0f * c;
    if (!(disc > 0.0f)) return false;
    float ds = sqrtf(disc);
    float q = b < 0.0f ? (-b - ds) / 2.0f : (-b + ds) / 2.0f;
    float t0 = q, t1 = c / q;
    float mn = fminf(t0, t1), mx = fmaxf(t0, t1);
    t = mn < 0.0f ? mx : mn;
    return t >= 0.0f;
}

// QuadDetail.h:21-57 (check_extent) and PlaneDetail.h:19-46
__device__ __forceinline__ bool isect_quad(float4 q0, float4 q1, float4 q2, float4 q3, f3 o, f3 d, float& t) {
    f3 n = xyz(q1);
    float OdotN = dot(o, n);
    float DdotN = dot(d, n);
    if (feq0(DdotN)) return false;
    t = (q1.w - OdotN) / DdotN;
    if (t < 0.0f) return false;
    f3 I = o + t * d;
    f3 r = I - xyz(q0);
    float x = dot(r, xyz(q2));
    float y = dot(r, xyz(q3));
    float s1 = q2.w, s2 = q3.w;
    return !(x < -s1 || x > s1 || y < -s2 || y > s2);
}
__device__ __forceinline__ bool isect_plane(float4 p0, float4 p1, f3 o, f3 d, float& t) {
    f3 n = xyz(p1);
    float PdotN = dot(xyz(p0), n);
    float OdotN = dot(o, n);
    float DdotN = dot(d, n);
    if (feq0(DdotN)) return false;
    t = (PdotN - OdotN) / DdotN;
    return !(t < 0.0f);
}

// AABBDetail.h:18-50 on the object's own box
__device__ __forceinline__ bool ref_box_hit(float4 lo, float4 hi, f3 o, f3 d) {
    bool hit = true;
    float tmin = 0.0f, tmax = __int_as_float(0x7f800000);
    const float los[3] = {lo.x, lo.y, lo.z}, his[3] = {hi.x, hi.y, hi.z};
    const float os[3] = {o.x, o.y, o.z}, ds[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float invD = 1.0f / (ds[a] + CUPBR_EPS);
        float t0 = (los[a] - os[a]) * invD;
        float t1 = (his[a] - os[a]) * invD;
        if (invD < 0.0f) { float tt = t0; t0 = t1; t1 = tt; }
        tmin = t0 > tmin ? t0 : tmin;
        tmax = t1 < tmax ? t1 : tmax;
        if (tmax <= tmin) hit = false;
    }
    return hit;
}

// Per-ray cache of the reference box predicate for the last object asked.
struct RefBoxCache {
    int32_t obj = -1;
    bool ok = true;
    __device__ __forceinline__ bool test(const DeviceScene& S, int32_t o_id, f3 o, f3 d) {
        if (o_id == obj) return ok;
        obj = o_id;
        float4 lo = __ldg(&S.objects[o_id].lo);
        if (lo.w == 0.0f) { ok = true; return true; }
        float4 hi = __ldg(&S.objects[o_id].hi);
        ok = ref_box_hit(lo, hi, o, d);
        return ok;
    }
};

struct TraceCounters {
    uint32_t nodes = 0, tris = 0;
};

// Normal and object of a closest-hit primitive at the hit point P
// (TriangleDetail.h:52, SphereDetail.h:64, QuadDetail.h:50, PlaneDetail.h:40).
__device__ __forceinline__ void hit_normal(const DeviceScene& S, int32_t prim, f3 P, f3& N, int32_t& obj) {
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
}

// Tracing::traceRay(scene, ray, index) (TracingDetail.h:68-116): the one
// object's own intersection, no box test; a mesh keeps its first strictly
// nearer triangle (MeshDetail.h:28-35).  t = INF when nothing is hit.
__device__ __forceinline__ bool trace_object(const DeviceScene& S, int32_t obj, f3 o, f3 d, float& t, f3& N) {
    const int4 info = __ldg(&S.obj_info[obj]);
    const float INF = __int_as_float(0x7f800000);
    t = INF;
    switch (info.x) {
        case 3:
        case 4: {  // TRIANGLE, MESH
            bool any = false;
            for (int k = 0; k < info.z; ++k) {
                const uint32_t s = __ldg(&S.key_slot[info.y + k]);
                const float4* p = S.tris + 3 * (size_t)s;
                float tt;
                if (isect_tri(__ldg(p), __ldg(p + 1), __ldg(p + 2), o, d, tt) && tt < t) {
                    t = tt;
                    N = xyz(__ldg(&S.tri_n[s]));
                    any = true;
                }
            }
            return any;
        }
        case 0: {  // SPHERE
            const uint32_t s = __ldg(&S.key_slot[info.y]);
            float4 s0 = __ldg(&S.spheres[2 * (size_t)s]), s1 = __ldg(&S.spheres[2 * (size_t)s + 1]);
            float tt;
            if (!isect_sphere(s0, s1, o, d, tt)) return false;
            t = tt;
            N = normalize((o + tt * d) - xyz(s0));
            return true;
        }
        case 2: {  // QUAD
            const uint32_t s = __ldg(&S.key_slot[info.y]);
            const float4* p = S.quads + 4 * (size_t)s;
            float tt;
            if (!isect_quad(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3), o, d, tt)) return false;
            t = tt;
            N = xyz(__ldg(p + 1));
            return true;
        }
        default: {  // PLANE
            const uint32_t s = __ldg(&S.key_slot[info.y]);
            float4 p0 = __ldg(&S.planes[2 * (size_t)s]), p1 = __ldg(&S.planes[2 * (size_t)s + 1]);
            float tt;
            if (!isect_plane(p0, p1, o, d, tt)) return false;
            t = tt;
            N = xyz(p1);
            return true;
        }
    }
}

__device__ __forceinline__ float safe_inv(float v) {
    return 1.0f / (fabsf(v) > 1e-20f ? v : copysignf(1e-20f, v));
}

// Node fetch (the 7 used float4s of a 4-wide node, bvh_build.hpp): the
// first `nsm` nodes are staged in shared memory.
__device__ __forceinline__ void fetch_node(const DeviceScene& S, const float4* __restrict__ snodes, uint32_t nsm,
                                           int32_t idx, float4* nb) {
    if ((uint32_t)idx < nsm) {
        const float4* p = snodes + BVH_NODE_F4 * idx;
#pragma unroll
        for (int k = 0; k < 7; ++k) nb[k] = p[k];
    } else {
        const float4* p = S.nodes + BVH_NODE_F4 * (size_t)idx;
#pragma unroll
        for (int k = 0; k < 7; ++k) nb[k] = __ldg(p + k);
    }
}

// Slab tests of a 4-wide node's children (t in [0, lim], FMA form on the
// conservatively inflated boxes).  Returns false when no child is hit;
// otherwise `first` is the nearest child hit and the others are pushed
// far-to-near (the nearest of them on top), each with its entry distance.
// KEEP_T = false (occlusion rays, whose limit never shrinks, so every entry
// pushed stays within it): the entry distances are not stored and the
// children are visited in node order.
template <bool KEEP_T = true>
__device__ __forceinline__ bool visit4(const float4* nb, f3 idir, f3 ood, float lim, int32_t& first, int32_t* st_ref,
                                       float* st_t, int& sp, bool& overflow) {
    const float INF = __int_as_float(0x7f800000);
    const float lx[4] = {nb[0].x, nb[0].y, nb[0].z, nb[0].w}, hx[4] = {nb[1].x, nb[1].y, nb[1].z, nb[1].w};
    const float ly[4] = {nb[2].x, nb[2].y, nb[2].z, nb[2].w}, hy[4] = {nb[3].x, nb[3].y, nb[3].z, nb[3].w};
    const float lz[4] = {nb[4].x, nb[4].y, nb[4].z, nb[4].w}, hz[4] = {nb[5].x, nb[5].y, nb[5].z, nb[5].w};
    int32_t r0 = __float_as_int(nb[6].x), r1 = __float_as_int(nb[6].y), r2 = __float_as_int(nb[6].z),
            r3 = __float_as_int(nb[6].w);
    float key[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float x0 = __fmaf_rn(lx[k], idir.x, -ood.x), x1 = __fmaf_rn(hx[k], idir.x, -ood.x);
        const float y0 = __fmaf_rn(ly[k], idir.y, -ood.y), y1 = __fmaf_rn(hy[k], idir.y, -ood.y);
        const float z0 = __fmaf_rn(lz[k], idir.z, -ood.z), z1 = __fmaf_rn(hz[k], idir.z, -ood.z);
        const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.0f));
        const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), lim));
        key[k] = tn <= tf ? tn : INF;
    }
    // a missing child has an inverted box, which a min/max slab test could
    // still accept, so it is excluded by its reference
    if (r0 == BVH_EMPTY) key[0] = INF;
    if (r1 == BVH_EMPTY) key[1] = INF;
    if (r2 == BVH_EMPTY) key[2] = INF;
    if (r3 == BVH_EMPTY) key[3] = INF;
    if (!KEEP_T) {
        // occlusion rays: any counted hit ends the ray, so the children are
        // not ordered by entry distance (measured faster than near-first:
        // k_connect 0.726 -> 0.700 ms per 1080p frame of the heightfield);
        // the first accepted child is entered, the others pushed
        const int lowest = key[0] < INF ? 0 : key[1] < INF ? 1 : key[2] < INF ? 2 : key[3] < INF ? 3 : -1;
        if (lowest < 0) return false;
        const int32_t rr[4] = {r0, r1, r2, r3};
        first = rr[lowest];
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            if (k == lowest || !(key[k] < INF)) continue;
            if (sp < CUPBR_STACK_SIZE) st_ref[sp++] = rr[k];
            else overflow = true;
        }
        return true;
    }
    float k0 = key[0], k1 = key[1], k2 = key[2], k3 = key[3];
#define CUPBR_CSWAP(ka, ra, kb, rb)              \
    if (kb < ka) {                               \
        const float tk = ka; ka = kb; kb = tk;   \
        const int32_t tr = ra; ra = rb; rb = tr; \
    }
    CUPBR_CSWAP(k0, r0, k1, r1)
    CUPBR_CSWAP(k2, r2, k3, r3)
    CUPBR_CSWAP(k0, r0, k2, r2)
    CUPBR_CSWAP(k1, r1, k3, r3)
    CUPBR_CSWAP(k1, r1, k2, r2)
#undef CUPBR_CSWAP
    if (!(k0 < INF)) return false;
    first = r0;
    const float ks[3] = {k3, k2, k1};
    const int32_t rs[3] = {r3, r2, r1};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!(ks[k] < INF)) continue;
        if (sp < CUPBR_STACK_SIZE) {
            st_ref[sp] = rs[k];
            if (KEEP_T) st_t[sp] = ks[k];
            ++sp;
        } else {
            overflow = true;
        }
    }
    return true;
}

// Closest hit (ANY = false) or visibility (ANY = true).
//   closest: on return t_best / best_prim / best_key hold the winning hit
//            (t_best = INF, best_prim = HIT_NONE when nothing is hit).
//   any    : returns true when some counted hit has t <= t_limit.
// `overflow` is set when the traversal stack would overflow (the entry is
// dropped; the caller reports it as an error).
// trace_scene_rt takes ANY / COUNT at run time, for kernels that trace
// closest-hit and shadow rays from one call site (one copy of the loop in
// the instruction cache); with constant flags it folds to trace_scene.
__device__ __forceinline__ bool trace_scene_rt(bool ANY, bool COUNT, const DeviceScene& S,
                                               const float4* __restrict__ snodes, uint32_t nsm, f3 o, f3 d,
                                               float t_limit, float& t_best, int32_t& best_prim, uint32_t& best_key,
                                               bool& overflow, TraceCounters& ctr) {
    RefBoxCache cache;
    t_best = ANY ? t_limit : __int_as_float(0x7f800000);
    best_prim = HIT_NONE;
    best_key = 0xFFFFFFFFu;

    // unbounded primitives (planes) are tested for every ray
    for (uint32_t i = 0; i < S.n_planes; ++i) {
        float4 p0 = __ldg(&S.planes[2 * i]), p1 = __ldg(&S.planes[2 * i + 1]);
        float t;
        if (isect_plane(p0, p1, o, d, t)) {
            uint32_t key = __float_as_uint(p0.w);
            if (ANY) {
                if (t <= t_limit) return true;
            } else if (t < t_best || (t == t_best && key < best_key)) {
                t_best = t; best_prim = prim_ref(3, i); best_key = key;
            }
        }
    }
    if (S.n_nodes == 0) return ANY ? false : best_prim != HIT_NONE;

    const f3 idir = mk(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    const f3 ood = mk(o.x * idir.x, o.y * idir.y, o.z * idir.z);

    int32_t st_ref[CUPBR_STACK_SIZE];
    float st_t[CUPBR_STACK_SIZE];
    int sp = 0;
    int32_t cur = 0;
    // A well-formed tree visits every node at most once per ray; the bound
    // turns a malformed node array into a reported error instead of a hang.
    uint32_t guard = 2u * S.n_nodes + 64u;

    for (;;) {
        if (--guard == 0u) {
            overflow = true;
            return ANY ? false : best_prim != HIT_NONE;
        }
        if (cur >= 0) {
            if ((uint32_t)cur >= S.n_nodes) {  // corrupt reference: report and stop
                overflow = true;
                return ANY ? false : best_prim != HIT_NONE;
            }
            float4 nb[7];
            fetch_node(S, snodes, nsm, cur, nb);
            if (COUNT) ctr.nodes++;
            int32_t first;
            if (visit4(nb, idir, ood, t_best, first, st_ref, st_t, sp, overflow)) {
                cur = first;
                continue;
            }
        } else {
            const uint32_t v = ~(uint32_t)cur;
            const uint32_t start = v >> 3, cnt = (v & 7u) + 1u;
            if (start < S.sphere_base) {
                for (uint32_t k = 0; k < cnt; ++k) {
                    const uint32_t s = start + k;
                    const float4* p = S.tris + 3 * (size_t)s;
                    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
                    if (COUNT) ctr.tris++;
                    float t;
                    if (!isect_tri(a, b, c, o, d, t)) continue;
                    const int32_t obj = __float_as_int(b.w);
                    if (ANY) {
                        if (t <= t_limit && cache.test(S, obj, o, d)) return true;
                    } else {
                        const uint32_t key = __float_as_uint(a.w);
                        if ((t < t_best || (t == t_best && key < best_key)) && cache.test(S, obj, o, d)) {
                            t_best = t; best_prim = prim_ref(0, s); best_key = key;
                        }
                    }
                }
            } else if (start < S.quad_base) {
                for (uint32_t k = 0; k < cnt; ++k) {
                    const uint32_t s = start + k - S.sphere_base;
                    float4 s0 = __ldg(&S.spheres[2 * (size_t)s]), s1 = __ldg(&S.spheres[2 * (size_t)s + 1]);
                    float t;
                    if (!isect_sphere(s0, s1, o, d, t)) continue;
                    const int32_t obj = __float_as_int(s1.z);
                    if (ANY) {
                        if (t <= t_limit && cache.test(S, obj, o, d)) return true;
                    } else {
                        const uint32_t key = __float_as_uint(s0.w);
                        if ((t < t_best || (t == t_best && key < best_key)) && cache.test(S, obj, o, d)) {
                            t_best = t; best_prim = prim_ref(1, s); best_key = key;
                        }
                    }
                }
            } else {
                for (uint32_t k = 0; k < cnt; ++k) {
                    const uint32_t s = start + k - S.quad_base;
                    const float4* p = S.quads + 4 * (size_t)s;
                    float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
                    float t;
                    if (COUNT) ctr.tris++;
                    if (!isect_quad(q0, q1, q2, q3, o, d, t)) continue;
                    if (ANY) {
                        if (t <= t_limit) return true;
                    } else {
                        const uint32_t key = __float_as_uint(q0.w);
                        if (t < t_best || (t == t_best && key < best_key)) {
                            t_best = t; best_prim = prim_ref(2, s); best_key = key;
                        }
                    }
                }
            }
        }
        // pop the next entry that can still hold a counted hit
        for (;;) {
            if (sp == 0) return ANY ? false : best_prim != HIT_NONE;
            --sp;
            if (st_t[sp] <= t_best) { cur = st_ref[sp]; break; }
        }
    }
}

template <bool ANY, bool COUNT>
__device__ __forceinline__ bool trace_scene(const DeviceScene& S, const float4* __restrict__ snodes, uint32_t nsm,
                                            f3 o, f3 d, float t_limit, float& t_best, int32_t& best_prim,
                                            uint32_t& best_key, bool& overflow, TraceCounters& ctr) {
    return trace_scene_rt(ANY, COUNT, S, snodes, nsm, o, d, t_limit, t_best, best_prim, best_key, overflow, ctr);
}

// ------------------------------------------------ resumable traversal ---
// State of one ray's traversal, so a persistent warp can run a bounded
// number of steps, hand finished lanes a new ray, and resume the others
// (dynamic ray fetch).  Same tests and acceptance rules as trace_scene.
struct TravState {
    f3 o, d, idir, ood;
    float t_limit, t_best;
    int32_t best_prim;
    uint32_t best_key;
    int32_t cur;
    int sp;
    uint32_t guard;
    bool done, hit;
    RefBoxCache cache;
};

template <bool ANY>
__device__ __forceinline__ void trav_init(const DeviceScene& S, TravState& s, f3 o, f3 d, float t_limit) {
    s.o = o;
    s.d = d;
    s.idir = mk(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    s.ood = mk(o.x * s.idir.x, o.y * s.idir.y, o.z * s.idir.z);
    s.t_limit = t_limit;
    s.t_best = ANY ? t_limit : __int_as_float(0x7f800000);
    s.best_prim = HIT_NONE;
    s.best_key = 0xFFFFFFFFu;
    s.cur = 0;
    s.sp = 0;
    s.guard = 2u * S.n_nodes + 64u;
    s.done = false;
    s.hit = false;
    s.cache.obj = -1;
    s.cache.ok = true;
    for (uint32_t i = 0; i < S.n_planes; ++i) {
        float4 p0 = __ldg(&S.planes[2 * i]), p1 = __ldg(&S.planes[2 * i + 1]);
        float t;
        if (isect_plane(p0, p1, o, d, t)) {
            uint32_t key = __float_as_uint(p0.w);
            if (ANY) {
                if (t <= t_limit) { s.hit = true; s.done = true; return; }
            } else if (t < s.t_best || (t == s.t_best && key < s.best_key)) {
                s.t_best = t; s.best_prim = prim_ref(3, i); s.best_key = key;
            }
        }
    }
    if (S.n_nodes == 0) s.done = true;
}

// Pops the next entry that can still hold a counted hit; false when empty.
// CHECK_T = false (occlusion rays): every entry can, none is skipped.
template <bool CHECK_T = true>
__device__ __forceinline__ bool trav_pop(TravState& s, const int32_t* st_ref, const float* st_t) {
    if (!CHECK_T) {
        if (s.sp == 0) return false;
        s.cur = st_ref[--s.sp];
        return true;
    }
    while (s.sp > 0) {
        --s.sp;
        if (st_t[s.sp] <= s.t_best) { s.cur = st_ref[s.sp]; return true; }
    }
    return false;
}

// Closest-hit test of the primitives of leaf v (packed start << 3 |
// count - 1) against the ray of s, with trav_run's acceptance rules (the
// packet traversal's leaf phase; trav_run keeps its own copy, which
// compiles to faster any-hit code than a shared helper did).
__device__ __forceinline__ void trav_leaf_closest(const DeviceScene& S, TravState& s, uint32_t v) {
    const uint32_t start = v >> 3, cnt = (v & 7u) + 1u;
    const f3 o = s.o, d = s.d;
    if (start < S.sphere_base) {
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t sl = start + k;
            const float4* p = S.tris + 3 * (size_t)sl;
            float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
            float t;
            if (!isect_tri(a, b, c, o, d, t)) continue;
            const uint32_t key = __float_as_uint(a.w);
            if ((t < s.t_best || (t == s.t_best && key < s.best_key)) && s.cache.test(S, __float_as_int(b.w), o, d)) {
                s.t_best = t; s.best_prim = prim_ref(0, sl); s.best_key = key;
            }
        }
    } else if (start < S.quad_base) {
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t sl = start + k - S.sphere_base;
            float4 s0 = __ldg(&S.spheres[2 * (size_t)sl]), s1 = __ldg(&S.spheres[2 * (size_t)sl + 1]);
            float t;
            if (!isect_sphere(s0, s1, o, d, t)) continue;
            const uint32_t key = __float_as_uint(s0.w);
            if ((t < s.t_best || (t == s.t_best && key < s.best_key)) && s.cache.test(S, __float_as_int(s1.z), o, d)) {
                s.t_best = t; s.best_prim = prim_ref(1, sl); s.best_key = key;
            }
        }
    } else {
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t sl = start + k - S.quad_base;
            const float4* p = S.quads + 4 * (size_t)sl;
            float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
            float t;
            if (!isect_quad(q0, q1, q2, q3, o, d, t)) continue;
            const uint32_t key = __float_as_uint(q0.w);
            if (t < s.t_best || (t == s.t_best && key < s.best_key)) {
                s.t_best = t; s.best_prim = prim_ref(2, sl); s.best_key = key;
            }
        }
    }
}

// Runs up to `rounds` rounds of (descend through inner nodes until a leaf,
// test that leaf); lanes that are on inner nodes and lanes that are at a
// leaf therefore execute their phases together (while-while).  Returns with
// s.done set when the ray is finished.
template <bool ANY, bool COUNT>
__device__ __forceinline__ void trav_run(const DeviceScene& S, const float4* __restrict__ snodes, uint32_t nsm,
                                         TravState& s, int32_t* st_ref, float* st_t, int rounds, bool& overflow,
                                         TraceCounters& ctr) {
    while (!s.done && rounds-- > 0) {
        // inner phase
        while (s.cur >= 0) {
            if (--s.guard == 0u || (uint32_t)s.cur >= S.n_nodes) { overflow = true; s.done = true; return; }
            float4 nb[7];
            fetch_node(S, snodes, nsm, s.cur, nb);
            if (COUNT) ctr.nodes++;
            int32_t first;
            if (visit4<!ANY>(nb, s.idir, s.ood, s.t_best, first, st_ref, st_t, s.sp, overflow)) {
                s.cur = first;
            } else if (!trav_pop<!ANY>(s, st_ref, st_t)) {
                s.done = true;
                return;
            }
        }
        // leaf phase
        const uint32_t v = ~(uint32_t)s.cur;
        const uint32_t start = v >> 3, cnt = (v & 7u) + 1u;
        const f3 o = s.o, d = s.d;
        if (start < S.sphere_base) {
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t sl = start + k;
                const float4* p = S.tris + 3 * (size_t)sl;
                float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
                if (COUNT) ctr.tris++;
                float t;
                if (!isect_tri(a, b, c, o, d, t)) continue;
                const int32_t obj = __float_as_int(b.w);
                if (ANY) {
                    if (t <= s.t_limit && s.cache.test(S, obj, o, d)) { s.hit = true; s.done = true; return; }
                } else {
                    const uint32_t key = __float_as_uint(a.w);
                    if ((t < s.t_best || (t == s.t_best && key < s.best_key)) && s.cache.test(S, obj, o, d)) {
                        s.t_best = t; s.best_prim = prim_ref(0, sl); s.best_key = key;
                    }
                }
            }
        } else if (start < S.quad_base) {
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t sl = start + k - S.sphere_base;
                float4 s0 = __ldg(&S.spheres[2 * (size_t)sl]), s1 = __ldg(&S.spheres[2 * (size_t)sl + 1]);
                if (COUNT) ctr.tris++;
                float t;
                if (!isect_sphere(s0, s1, o, d, t)) continue;
                const int32_t obj = __float_as_int(s1.z);
                if (ANY) {
                    if (t <= s.t_limit && s.cache.test(S, obj, o, d)) { s.hit = true; s.done = true; return; }
                } else {
                    const uint32_t key = __float_as_uint(s0.w);
                    if ((t < s.t_best || (t == s.t_best && key < s.best_key)) && s.cache.test(S, obj, o, d)) {
                        s.t_best = t; s.best_prim = prim_ref(1, sl); s.best_key = key;
                    }
                }
            }
        } else {
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t sl = start + k - S.quad_base;
                const float4* p = S.quads + 4 * (size_t)sl;
                float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
                if (COUNT) ctr.tris++;
                float t;
                if (!isect_quad(q0, q1, q2, q3, o, d, t)) continue;
                if (ANY) {
                    if (t <= s.t_limit) { s.hit = true; s.done = true; return; }
                } else {
                    const uint32_t key = __float_as_uint(q0.w);
                    if (t < s.t_best || (t == s.t_best && key < s.best_key)) {
                        s.t_best = t; s.best_prim = prim_ref(2, sl); s.best_key = key;
                    }
                }
            }
        }
        if (!trav_pop<!ANY>(s, st_ref, st_t)) { s.done = true; return; }
    }
}

// ------------------------------------------------------ warp packets ---
// Coherent rays (a warp's camera rays over one pixel tile) walk the tree
// as one packet: the node sequence, the stack pointer and the node refs
// are the same in every lane, each lane keeps its own ray, entry
// distances and closest hit.  A child is visited when any lane's slab test
// accepts it, nearest first by the smallest entry distance over the lanes;
// a stack entry is resumed while any lane's own entry distance is still
// within its closest hit.  Because the builder inflated every box
// conservatively, a box that holds a primitive is never entered later than
// that primitive's hit distance, so a ray's closest hit does not depend on
// the order in which nodes are visited and extra leaves tested for other
// lanes cannot change it: each lane ends with the same hit as trace_scene.

// Slab tests of a 4-wide node for every lane (as visit4).  Returns false
// when no lane hits a child; otherwise `first` is the child with the
// nearest entry over the lanes and the other accepted children are pushed
// far-to-near with each lane's own entry distance (INF where it missed).
__device__ __forceinline__ bool packet_visit4(const float4* nb, f3 idir, f3 ood, float lim, int32_t& first,
                                              int32_t* st_ref, float* st_t, int& sp, bool& overflow) {
    const unsigned full = 0xffffffffu;
    const float INF = __int_as_float(0x7f800000);
    const float lx[4] = {nb[0].x, nb[0].y, nb[0].z, nb[0].w}, hx[4] = {nb[1].x, nb[1].y, nb[1].z, nb[1].w};
    const float ly[4] = {nb[2].x, nb[2].y, nb[2].z, nb[2].w}, hy[4] = {nb[3].x, nb[3].y, nb[3].z, nb[3].w};
    const float lz[4] = {nb[4].x, nb[4].y, nb[4].z, nb[4].w}, hz[4] = {nb[5].x, nb[5].y, nb[5].z, nb[5].w};
    int32_t r[4] = {__float_as_int(nb[6].x), __float_as_int(nb[6].y), __float_as_int(nb[6].z),
                    __float_as_int(nb[6].w)};
    float key[4];
    uint32_t wk[4];  // nearest entry over the lanes, as ordered bits (INF: no lane)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float x0 = __fmaf_rn(lx[k], idir.x, -ood.x), x1 = __fmaf_rn(hx[k], idir.x, -ood.x);
        const float y0 = __fmaf_rn(ly[k], idir.y, -ood.y), y1 = __fmaf_rn(hy[k], idir.y, -ood.y);
        const float z0 = __fmaf_rn(lz[k], idir.z, -ood.z), z1 = __fmaf_rn(hz[k], idir.z, -ood.z);
        const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.0f));
        const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), lim));
        key[k] = (tn <= tf && r[k] != BVH_EMPTY) ? tn : INF;
        // entry distances are >= 0 (a -0 clears to 0), so their bits order as the values
        wk[k] = __reduce_min_sync(full, __float_as_uint(key[k]) & 0x7fffffffu);
    }
#define CUPBR_PSWAP(a, b)                                                                \
    if (wk[b] < wk[a]) {                                                                 \
        const uint32_t tw = wk[a]; wk[a] = wk[b]; wk[b] = tw;                            \
        const float tk = key[a]; key[a] = key[b]; key[b] = tk;                           \
        const int32_t tr = r[a]; r[a] = r[b]; r[b] = tr;                                 \
    }
    CUPBR_PSWAP(0, 1)
    CUPBR_PSWAP(2, 3)
    CUPBR_PSWAP(0, 2)
    CUPBR_PSWAP(1, 3)
    CUPBR_PSWAP(1, 2)
#undef CUPBR_PSWAP
    const uint32_t inf_bits = 0x7f800000u;
    if (wk[0] >= inf_bits) return false;
    first = r[0];
#pragma unroll
    for (int k = 3; k >= 1; --k) {
        if (wk[k] >= inf_bits) continue;
        if (sp < CUPBR_STACK_SIZE) {
            st_ref[sp] = r[k];
            st_t[sp] = key[k];
            ++sp;
        } else {
            overflow = true;
        }
    }
    return true;
}

// Resumes the top stack entry that some lane can still use; false when the
// stack is empty.
__device__ __forceinline__ bool packet_pop(float t_best, const int32_t* st_ref, const float* st_t, int& sp,
                                           int32_t& cur) {
    while (sp > 0) {
        --sp;
        if (__any_sync(0xffffffffu, st_t[sp] <= t_best)) {
            cur = st_ref[sp];
            return true;
        }
    }
    return false;
}

}  // namespace cupbr_b200
