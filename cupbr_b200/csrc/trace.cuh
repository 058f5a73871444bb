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

#include "dev_common.cuh"

namespace cupbr_b200 {

#ifndef CUPBR_STACK_SIZE
#define CUPBR_STACK_SIZE 48
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

// Node fetch: the first `nsm` nodes are staged in shared memory.
__device__ __forceinline__ void fetch_node(const DeviceScene& S, const float4* __restrict__ snodes, uint32_t nsm,
                                           int32_t idx, float4& n0, float4& n1, float4& n2, float4& n3) {
    if ((uint32_t)idx < nsm) {
        const float4* p = snodes + 4 * idx;
        n0 = p[0]; n1 = p[1]; n2 = p[2]; n3 = p[3];
    } else {
        const float4* p = S.nodes + 4 * (size_t)idx;
        n0 = __ldg(p); n1 = __ldg(p + 1); n2 = __ldg(p + 2); n3 = __ldg(p + 3);
    }
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
            float4 n0, n1, n2, n3;
            fetch_node(S, snodes, nsm, cur, n0, n1, n2, n3);
            if (COUNT) ctr.nodes++;
            const float lim = t_best;
            float a0 = __fmaf_rn(n0.x, idir.x, -ood.x), a1 = __fmaf_rn(n0.y, idir.x, -ood.x);
            float b0 = __fmaf_rn(n0.z, idir.y, -ood.y), b1 = __fmaf_rn(n0.w, idir.y, -ood.y);
            float c0 = __fmaf_rn(n2.x, idir.z, -ood.z), c1 = __fmaf_rn(n2.y, idir.z, -ood.z);
            float tn0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), 0.0f));
            float tf0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), lim));
            float d0 = __fmaf_rn(n1.x, idir.x, -ood.x), d1 = __fmaf_rn(n1.y, idir.x, -ood.x);
            float e0 = __fmaf_rn(n1.z, idir.y, -ood.y), e1 = __fmaf_rn(n1.w, idir.y, -ood.y);
            float f0 = __fmaf_rn(n2.z, idir.z, -ood.z), f1 = __fmaf_rn(n2.w, idir.z, -ood.z);
            float tn1 = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), 0.0f));
            float tf1 = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fminf(fmaxf(f0, f1), lim));
            int32_t ch0 = __float_as_int(n3.x), ch1 = __float_as_int(n3.y);
            // a missing child has an inverted box, which a min/max slab test
            // would still accept, so it is excluded by its reference
            bool h0 = tn0 <= tf0 && ch0 != (int32_t)0x80000000;
            bool h1 = tn1 <= tf1 && ch1 != (int32_t)0x80000000;
            if (h0 && h1) {
                bool sw = tn1 < tn0;
                int32_t nr = sw ? ch1 : ch0, fr = sw ? ch0 : ch1;
                float tfar = sw ? tn0 : tn1;
                if (sp < CUPBR_STACK_SIZE) { st_ref[sp] = fr; st_t[sp] = tfar; ++sp; }
                else overflow = true;
                cur = nr;
                continue;
            }
            if (h0) { cur = ch0; continue; }
            if (h1) { cur = ch1; continue; }
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
__device__ __forceinline__ bool trav_pop(TravState& s, const int32_t* st_ref, const float* st_t) {
    while (s.sp > 0) {
        --s.sp;
        if (st_t[s.sp] <= s.t_best) { s.cur = st_ref[s.sp]; return true; }
    }
    return false;
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
            float4 n0, n1, n2, n3;
            fetch_node(S, snodes, nsm, s.cur, n0, n1, n2, n3);
            if (COUNT) ctr.nodes++;
            const float lim = s.t_best;
            const f3 idir = s.idir, ood = s.ood;
            float a0 = __fmaf_rn(n0.x, idir.x, -ood.x), a1 = __fmaf_rn(n0.y, idir.x, -ood.x);
            float b0 = __fmaf_rn(n0.z, idir.y, -ood.y), b1 = __fmaf_rn(n0.w, idir.y, -ood.y);
            float c0 = __fmaf_rn(n2.x, idir.z, -ood.z), c1 = __fmaf_rn(n2.y, idir.z, -ood.z);
            float tn0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), 0.0f));
            float tf0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), lim));
            float d0 = __fmaf_rn(n1.x, idir.x, -ood.x), d1 = __fmaf_rn(n1.y, idir.x, -ood.x);
            float e0 = __fmaf_rn(n1.z, idir.y, -ood.y), e1 = __fmaf_rn(n1.w, idir.y, -ood.y);
            float f0 = __fmaf_rn(n2.z, idir.z, -ood.z), f1 = __fmaf_rn(n2.w, idir.z, -ood.z);
            float tn1 = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), 0.0f));
            float tf1 = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fminf(fmaxf(f0, f1), lim));
            int32_t ch0 = __float_as_int(n3.x), ch1 = __float_as_int(n3.y);
            bool h0 = tn0 <= tf0 && ch0 != (int32_t)0x80000000;
            bool h1 = tn1 <= tf1 && ch1 != (int32_t)0x80000000;
            if (h0 && h1) {
                bool sw = tn1 < tn0;
                if (s.sp < CUPBR_STACK_SIZE) {
                    st_ref[s.sp] = sw ? ch0 : ch1;
                    st_t[s.sp] = sw ? tn0 : tn1;
                    ++s.sp;
                } else {
                    overflow = true;
                }
                s.cur = sw ? ch1 : ch0;
            } else if (h0) {
                s.cur = ch0;
            } else if (h1) {
                s.cur = ch1;
            } else if (!trav_pop(s, st_ref, st_t)) {
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
        if (!trav_pop(s, st_ref, st_t)) { s.done = true; return; }
    }
}

}  // namespace cupbr_b200
