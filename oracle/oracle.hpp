// CPU oracle for the cupbr rendering hot path -- TEST INFRASTRUCTURE ONLY.
//
// This header restates, in plain C++ templated on the arithmetic type R
// (float for reference-semantics parity, double for converged FP64 images),
// the algorithms of cupbr's path-tracing path.  It is the checker for the
// CUDA kernels in cupbr_b200/csrc: only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg may load it.  Nothing in the product links it.
//
// Every function cites the reference file:line it restates (paths are
// relative to the cupbr project root).  In float mode the operation order of
// every +,-,*,/ and sqrt follows the reference exactly and the build uses
// -ffp-contract=off, so results are bit-identical to the reference's own
// __host__ __device__ code compiled for the host (which is how the golden
// vectors under tests/golden/ were produced, see oracle/ref_host.cpp).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- vectors ---
// lib/include/Math/VectorTypes.h, lib/src/Math/VectorOperationsDetail.h
template <typename R>
struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    explicit V3(R v) : x(v), y(v), z(v) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <typename R> inline V3<R> operator+(const V3<R>& a, const V3<R>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> inline V3<R> operator-(const V3<R>& a, const V3<R>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// VectorOperationsDetail.h:112-116  (scalar * vector)
template <typename R> inline V3<R> operator*(R s, const V3<R>& v) { return {s * v.x, s * v.y, s * v.z}; }
// VectorOperationsDetail.h:105-108  (vector * scalar forwards to scalar * vector)
template <typename R> inline V3<R> operator*(const V3<R>& v, R s) { return {s * v.x, s * v.y, s * v.z}; }
template <typename R> inline V3<R> operator*(const V3<R>& a, const V3<R>& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <typename R> inline V3<R> operator/(const V3<R>& v, R s) { return {v.x / s, v.y / s, v.z / s}; }
template <typename R> inline void operator+=(V3<R>& a, const V3<R>& b) { a.x += b.x; a.y += b.y; a.z += b.z; }

template <typename R> struct V4 { R x, y, z, w; };

template <typename R> inline R sqrt_(R v) { return std::sqrt(v); }

// lib/src/Math/VectorFunctionsDetail.h:48-79
template <typename R> inline R dot(const V3<R>& v, const V3<R>& w) { return v.x * w.x + v.y * w.y + v.z * w.z; }
template <typename R> inline R norm(const V3<R>& v) { return sqrt_(dot(v, v)); }
template <typename R> inline V3<R> normalize(const V3<R>& v) { return v / norm(v); }
template <typename R> inline V3<R> cross(const V3<R>& v, const V3<R>& w) {
    return {v.y * w.z - v.z * w.y, v.z * w.x - v.x * w.z, v.x * w.y - v.y * w.x};
}
template <typename R> inline V3<R> vexp(const V3<R>& v) { return {std::exp(v.x), std::exp(v.y), std::exp(v.z)}; }

template <typename R> inline R eps() { return R(1e-5f); }   // lib/include/Math/Functions.h:4
template <typename R> inline R inf() { return std::numeric_limits<R>::infinity(); }

// ------------------------------------------------------------------ math ---
// lib/src/Math/FunctionsDetail.h:10-15
template <typename R> inline bool safeFloatEqual(R lhs, R rhs, R e = eps<R>()) { return std::abs(lhs - rhs) < e; }
// FunctionsDetail.h:17-22
template <typename R> inline R clampR(R x, R lo, R hi) { return std::fmin(std::fmax(x, lo), hi); }
// FunctionsDetail.h:24-29
template <typename R> inline R delta(R inp) { return safeFloatEqual(inp, R(0)) ? R(1) : R(0); }
// FunctionsDetail.h:31-36
template <typename R> inline V3<R> reflect(const V3<R>& inc, const V3<R>& n) {
    return normalize((R(2) * dot(inc, n)) * n - inc);
}
// FunctionsDetail.h:38-52
template <typename R> inline V3<R> refract(R eta, const V3<R>& inc, const V3<R>& n) {
    R NdotI = dot(inc, n);
    R k = R(1) - eta * eta * (R(1) - NdotI * NdotI);
    if (k < 0) return V3<R>(R(0));
    return (-eta) * inc - ((-eta) * NdotI + sqrt_(k)) * n;
}
// FunctionsDetail.h:54-60
template <typename R> inline R fresnel(R F0, R VdotH) {
    R p = std::fmax(R(0), R(1) - VdotH);
    return F0 + (R(1) - F0) * p * p * p * p * p;
}
// FunctionsDetail.h:62-68
template <typename R> inline V3<R> fresnel(const V3<R>& F0, R VdotH) {
    R p = std::fmax(R(0), R(1) - VdotH);
    return F0 + (V3<R>(R(1)) - F0) * p * p * p * p * p;
}
// FunctionsDetail.h:70-87  (4-round TEA seed hash)
inline uint32_t tea4(uint32_t val0, uint32_t val1) {
    uint32_t v0 = val0, v1 = val1, s0 = 0;
    for (uint32_t n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
// FunctionsDetail.h:89-98  (LCG; the draw is always produced in float)
template <typename R> inline R rnd(uint32_t& prev) {
    prev = 1664525u * prev + 1013904223u;
    return R((float)(prev & 0x00FFFFFFu) / (float)0x01000000);
}
// FunctionsDetail.h:100-117
template <typename R> inline V3<R> toLocalFrame(const V3<R>& N, const V3<R>& d) {
    const R x = N.x, y = N.y, z = N.z;
    const R sz = (z >= R(0)) ? R(1) : R(-1);
    const R a = R(1) / (sz + z);
    const R ya = y * a;
    const R b = x * ya;
    const R c = x * sz;
    V3<R> lx(c * x * a - R(1), sz * b, c);
    V3<R> ly(b, y * ya - sz, y);
    return d.x * lx + d.y * ly + d.z * N;
}

template <typename R> inline R pif() { return R(static_cast<float>(M_PI)); }

// -------------------------------------------------------------- material ---
// lib/include/Geometry/Material.h:14-178, lib/include/DataStructure/Volume.h:9-21
enum MatType { LAMBERT = 0, PHONG = 1, MIRROR = 2, GLASS = 3, GGX = 4, VOLUME = 5 };

template <typename R>
struct Material {
    V3<R> albedo_e{R(0)}, albedo_d{R(1)}, albedo_s{R(0)};
    R shininess = R(128.0f * 0.4f), roughness = R(1), eta = R(1.5f);
    V3<R> sigma_s{R(1)}, sigma_a{R(1)};
    R g = R(0);
    int interface_glass = 0;
    int type = LAMBERT;
};

// MaterialDetail.h:13-18
template <typename R> inline R D_GGX(R NdotH, R roughness) {
    R a2 = roughness * roughness;
    R d = (NdotH * a2 - NdotH) * NdotH + R(1);
    return a2 / (pif<R>() * d * d);
}
// MaterialDetail.h:20-31
template <typename R> inline R V_SmithJointGGX(R NdotL, R NdotV, R roughness) {
    R a2 = roughness * roughness;
    R denomA = NdotV * sqrt_(a2 + (R(1) - a2) * NdotL * NdotL);
    R denomB = NdotL * sqrt_(a2 + (R(1) - a2) * NdotV * NdotV);
    R G = R(2) * NdotL * NdotV / (denomA + denomB + eps<R>());
    return G / (R(4) * NdotV * NdotL + eps<R>());
}

// MaterialDetail.h:209-215
template <typename R> inline V3<R> brdf_lambert(const Material<R>& m) { return m.albedo_d / pif<R>(); }
template <typename R> inline V3<R> brdf_phong(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    V3<R> h = normalize(inc + out);
    return m.albedo_s * R(std::pow(std::fmax(R(0), dot(h, n)), m.shininess));
}
// MaterialDetail.h:217-223
template <typename R> inline V3<R> brdf_mirror(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    V3<R> r = reflect(inc, n);
    return m.albedo_s * delta(R(1) - dot(out, r)) / dot(out, n);
}
// MaterialDetail.h:225-257
template <typename R> inline V3<R> btdf_glass(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    if (dot(inc, n) * dot(out, n) > 0) {
        if (dot(inc, n) > 0) return brdf_mirror(m, inc, out, n);
        return brdf_mirror(m, inc, out, R(-1) * n);
    }
    V3<R> refracted;
    V3<R> nn = n;
    if (dot(inc, n) > 0) {
        refracted = refract(R(1) / m.eta, inc, n);
    } else {
        refracted = refract(m.eta, inc, R(-1) * n);
        nn = R(-1) * n;
    }
    return m.albedo_s * delta(R(1) - dot(refracted, out)) / dot(inc, nn);
}
// MaterialDetail.h:259-274
template <typename R> inline V3<R> brdf_ggx(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    V3<R> H = normalize(inc + out);
    R NdotH = dot(n, H), LdotH = dot(out, H), NdotL = dot(n, out), NdotV = dot(n, inc);
    R ndf = D_GGX(NdotH, m.roughness);
    R vis = V_SmithJointGGX(NdotL, NdotV, m.roughness);
    return ndf * vis * fresnel(m.albedo_s, LdotH);
}
// MaterialDetail.h:35-74
template <typename R> inline V3<R> brdf(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    switch (m.type) {
        case LAMBERT: return brdf_lambert(m);
        case PHONG: return brdf_phong(m, inc, out, n) + brdf_lambert(m);
        case MIRROR: return brdf_mirror(m, inc, out, n);
        case GLASS: return btdf_glass(m, inc, out, n);
        case GGX: return brdf_ggx(m, inc, out, n);
        default: return V3<R>(R(0));
    }
}

template <typename R> inline V4<R> mk4(const V3<R>& v, R w) { return {v.x, v.y, v.z, w}; }

// MaterialDetail.h:113-132
template <typename R> inline V4<R> sample_lambert(uint32_t& seed, const V3<R>& n) {
    const R xi1 = rnd<R>(seed);
    const R xi2 = rnd<R>(seed);
    const R r = sqrt_(xi1);
    const R phi = R(2.0f * 3.14159f) * xi2;
    const R x = r * std::cos(phi);
    const R y = r * std::sin(phi);
    const R z = sqrt_(std::fmax(R(0), R(1) - x * x - y * y));
    V3<R> d = normalize(toLocalFrame(n, V3<R>(x, y, z)));
    R p = std::fmax(eps<R>(), dot(d, n)) / R(3.14159f);
    return mk4(d, p);
}
// MaterialDetail.h:134-141
template <typename R> inline V4<R> sample_mirror(const V3<R>& inc, const V3<R>& n) { return mk4(reflect(inc, n), R(1)); }
// MaterialDetail.h:143-169
template <typename R> inline V4<R> sample_glass(const Material<R>& m, uint32_t& seed, const V3<R>& inc, const V3<R>& n0) {
    const R NdotV = dot(inc, n0);
    bool outside = NdotV > R(0);
    R e = outside ? R(1) / m.eta : m.eta;
    V3<R> n = outside ? n0 : R(-1) * n0;
    R F0 = (m.eta - R(1)) / (m.eta + R(1));
    F0 *= F0;
    R p_reflect = fresnel(F0, std::abs(dot(inc, n)));
    R xi = rnd<R>(seed);
    V3<R> refr = refract(e, inc, n);
    V3<R> d;
    if (xi <= p_reflect || safeFloatEqual(norm(refr), R(0))) d = reflect(inc, n);
    else d = normalize(refr);
    return mk4(d, R(1));
}
// MaterialDetail.h:171-200
template <typename R> inline V4<R> sample_ggx(const Material<R>& m, uint32_t& seed, const V3<R>& inc, const V3<R>& n) {
    R u = rnd<R>(seed);
    R v = rnd<R>(seed);
    R cosTheta = sqrt_((R(1) - u) / (R(1) + (m.roughness * m.roughness - R(1)) * u));
    R sinTheta = sqrt_(std::fmax(R(0), R(1) - cosTheta * cosTheta));
    R phi = R(2.0f * static_cast<float>(M_PI)) * v;
    R x = sinTheta * std::cos(phi);
    R y = sinTheta * std::sin(phi);
    R z = cosTheta;
    V3<R> H = toLocalFrame(n, V3<R>(x, y, z));
    V3<R> L = reflect(inc, H);
    R LdotH = dot(inc, H);
    R NdotH = dot(n, H);
    if (dot(n, L) <= R(0)) return {R(0), R(0), R(0), R(1)};
    R p = D_GGX(NdotH, m.roughness) * NdotH / std::abs(R(4) * LdotH);
    return mk4(L, p);
}
// MaterialDetail.h:76-111
template <typename R> inline V4<R> sampleDirection(const Material<R>& m, uint32_t& seed, const V3<R>& inc, const V3<R>& n) {
    switch (m.type) {
        case LAMBERT:
        case PHONG: return sample_lambert(seed, n);
        case MIRROR: return sample_mirror(inc, n);
        case GLASS: return sample_glass(m, seed, inc, n);
        case GGX: return sample_ggx(m, seed, inc, n);
        case VOLUME:
            return m.interface_glass ? sample_glass(m, seed, inc, n) : mk4(R(-1) * inc, R(1));
    }
    return {inf<R>(), inf<R>(), inf<R>(), inf<R>()};
}
// MaterialDetail.h:276-286
template <typename R> inline R hg_phase(R g, R cos_theta) {
    // the literal 0.25 is a double: the quotient is formed in double
    if (std::abs(g) < R(1e-3f)) return R(0.25 / double(pif<R>()));
    R g2 = g * g;
    R area = R(4.0f * 3.14159f);
    return (R(1) - g2) / area * R(std::pow(R(1) + g2 - R(2) * g * cos_theta, R(-1.5f)));
}
// MaterialDetail.h:288-313
template <typename R> inline V4<R> sample_hg(R g_, const V3<R>& forward, uint32_t& seed) {
    R g = g_ < R(0) ? std::fmin(R(-1e-3), g_) : std::fmax(R(1e-3), g_);
    R u1 = rnd<R>(seed);
    R u2 = rnd<R>(seed);
    R g2 = g * g;
    R d = (R(1) - g2) / (R(1) - g + R(2) * g * u1);
    R cos_theta = clampR(R(0.5f) / g * (R(1) + g2 - d * d), R(-1), R(1));
    R sin_theta = sqrt_(std::fmax(R(0), R(1) - cos_theta * cos_theta));
    R phi = R(2.0f * 3.14159f) * u2;
    R x = sin_theta * std::cos(phi);
    R y = sin_theta * std::sin(phi);
    R z = cos_theta;
    V3<R> res = normalize(toLocalFrame(forward, V3<R>(x, y, z)));
    R pdf = hg_phase(g, dot(forward, res));
    return mk4(res, pdf);
}

// ----------------------------------------------------------------- light ---
// lib/include/DataStructure/Light.h:20-71, lib/src/DataStructure/LightDetail.h:8-52
template <typename R>
struct Light {
    int type = 0;  // 0 = POINT, 1 = AREA
    V3<R> position, intensity, radiance, he1, he2;
};
template <typename R> inline V3<R> light_sample(const Light<R>& l, uint32_t& seed, const V3<R>& P, V3<R>& dir, R& dist) {
    if (l.type == 0) {  // LightDetail.h:23-30
        dir = normalize(l.position - P);
        dist = norm(l.position - P);
        return l.intensity / (dist * dist);
    }
    // LightDetail.h:32-52
    R xi1 = rnd<R>(seed) * R(2) - R(1);
    R xi2 = rnd<R>(seed) * R(2) - R(1);
    V3<R> s = l.position + xi1 * l.he1 + xi2 * l.he2;
    V3<R> n = normalize(cross(l.he1, l.he2));
    R area = R(4) * norm(l.he1) * norm(l.he2);
    dir = normalize(s - P);
    dist = norm(s - P);
    R NdotL = dot(dir, n);
    if (NdotL < 0) NdotL *= R(-1);
    R solidAngle = area * NdotL / (dist * dist);
    return l.radiance * solidAngle;
}

// -------------------------------------------------------------- geometry ---
enum GeoType { SPHERE = 0, PLANE = 1, QUAD = 2, TRIANGLE = 3, MESH = 4 };

template <typename R>
struct Ray {
    V3<R> o, d;
    // lib/src/Geometry/RayDetail.h:8-14: the constructor normalizes
    Ray(const V3<R>& origin, const V3<R>& dir) : o(origin), d(normalize(dir)) {}
};

template <typename R>
struct Hit {
    R depth = inf<R>();
    V3<R> P, N;
    int obj = -1;   // scene_index (object id)
    int tri = -1;   // triangle index inside a MESH / TRIANGLE object, -1 otherwise
};

template <typename R>
struct Tri { V3<R> v1, v2, v3, n; };

template <typename R>
struct Object {
    int type = MESH;
    Material<R> mat;
    V3<R> p0, p1, p2, p3;     // sphere: center, (r,_,_); plane: pos, normal; quad: pos, normal, e1, e2
    R radius = 0;
    std::vector<Tri<R>> tris; // MESH / TRIANGLE
    V3<R> box_lo{-inf<R>()}, box_hi{inf<R>()};  // Geometry.cu:6-10 default is infinite
    // albedo-texture binding (not in the reference): planar projection with
    // the axes pre-divided by their squared length (computed in float)
    bool textured = false;
    V3<R> tex_o{R(0)}, tex_u{R(0)}, tex_v{R(0)};
};

// TriangleDetail.h:11-19: normal computed at construction
template <typename R> inline Tri<R> make_tri(const V3<R>& a, const V3<R>& b, const V3<R>& c) {
    Tri<R> t;
    t.v1 = a; t.v2 = b; t.v3 = c;
    t.n = normalize(cross(b - a, c - a));
    return t;
}

// TriangleDetail.h:21-57 (Moller-Trumbore in the reference's operation order)
template <typename R> inline bool tri_hit(const Tri<R>& tr, const Ray<R>& ray, R& t_out) {
    V3<R> v0v1 = tr.v2 - tr.v1;
    V3<R> v0v2 = tr.v3 - tr.v1;
    V3<R> pvec = cross(ray.d, v0v2);
    R det = dot(v0v1, pvec);
    if (safeFloatEqual(det, R(0))) return false;
    R invDet = R(1) / det;
    V3<R> tvec = ray.o - tr.v1;
    R u = dot(tvec, pvec) * invDet;
    if (u < R(0) || u > R(1)) return false;
    V3<R> qvec = cross(tvec, v0v1);
    R v = dot(ray.d, qvec) * invDet;
    if (v < R(0) || u + v > R(1)) return false;
    R t = dot(v0v2, qvec) * invDet;
    if (t < R(0)) return false;
    t_out = t;
    return true;
}

// AABBDetail.h:18-50 (slab test with the +EPSILON direction perturbation)
template <typename R> inline bool ref_aabb_hit(const V3<R>& mn, const V3<R>& mx, const Ray<R>& ray) {
    bool hit = true;
    R t_min = 0, t_max = inf<R>();
    for (int a = 0; a < 3; ++a) {
        R invD = R(1) / (ray.d[a] + eps<R>());
        R t0 = (mn[a] - ray.o[a]) * invD;
        R t1 = (mx[a] - ray.o[a]) * invD;
        if (invD < R(0)) std::swap(t0, t1);
        t_min = t0 > t_min ? t0 : t_min;
        t_max = t1 < t_max ? t1 : t_max;
        if (t_max <= t_min) hit = false;
    }
    return hit;
}

// Per-object intersection: SphereDetail.h:33-74, PlaneDetail.h:19-46,
// QuadDetail.h:21-57, TriangleDetail.h:21-57, MeshDetail.h:21-40.
template <typename R> inline Hit<R> object_hit(const Object<R>& ob, int id, const Ray<R>& ray) {
    Hit<R> g;
    switch (ob.type) {
        case SPHERE: {
            V3<R> OS = ray.o - ob.p0;
            R b = R(2) * dot(ray.d, OS);
            R c = dot(OS, OS) - ob.radius * ob.radius;
            R disc = b * b - R(4) * c;
            if (disc > 0) {
                R ds = sqrt_(disc);
                R q = b < 0 ? (-b - ds) / R(2) : (-b + ds) / R(2);
                R t0 = q, t1 = c / q;
                R mn = std::fmin(t0, t1), mx = std::fmax(t0, t1);
                R t = mn < 0 ? mx : mn;
                if (t >= 0) {
                    g.P = ray.o + t * ray.d;
                    g.depth = t;
                    g.N = normalize(g.P - ob.p0);
                    g.obj = id;
                }
            }
            return g;
        }
        case PLANE:
        case QUAD: {
            R PdotN = dot(ob.p0, ob.p1);
            R OdotN = dot(ray.o, ob.p1);
            R DdotN = dot(ray.d, ob.p1);
            if (safeFloatEqual(DdotN, R(0))) return g;
            R t = (PdotN - OdotN) / DdotN;
            if (t < 0) return g;
            V3<R> I = ray.o + t * ray.d;
            if (ob.type == QUAD) {
                R x = dot(I - ob.p0, ob.p2);
                R y = dot(I - ob.p0, ob.p3);
                R s1 = dot(ob.p2, ob.p2);
                R s2 = dot(ob.p3, ob.p3);
                if (x < -s1 || x > s1 || y < -s2 || y > s2) return g;
            }
            g.P = I;
            g.depth = t;
            g.N = ob.p1;
            g.obj = id;
            return g;
        }
        case TRIANGLE:
        case MESH: {
            // MeshDetail.h:28-35: first strictly-nearer triangle wins
            for (size_t i = 0; i < ob.tris.size(); ++i) {
                R t;
                if (tri_hit(ob.tris[i], ray, t) && t < g.depth) {
                    g.depth = t;
                    g.P = ray.o + t * ray.d;
                    g.N = ob.tris[i].n;
                    g.tri = (int)i;
                }
            }
            if (g.depth != inf<R>()) g.obj = id;
            return g;
        }
    }
    return g;
}

// ----------------------------------------------------------------- scene ---
template <typename R>
struct Scene {
    std::vector<Object<R>> objects;
    std::vector<Light<R>> lights;
    std::vector<V3<R>> env;  // lat-long RGB, row-major
    uint32_t env_w = 0, env_h = 0;
    V3<R> vol_sigma_s{R(1)}, vol_sigma_a{R(1)};  // Volume.h:17-20 defaults
    R vol_g = 0;
    std::vector<int> dfs_order;  // leaf order of the reference's object BVH

    // BoundingVolumeHierarchy.cpp:46-136: recursive median split of objects
    // by aabb().minimum().x (the axis expression (rand()/RAND_MAX)%3 is 0
    // except when rand() returns RAND_MAX), stable sort, leaves of 1 or 2
    // objects ordered by the comparator.  Traversal
    // (BoundingVolumeHierarchyDetail.h:11-101) is a left-first DFS that skips
    // subtrees whose box test fails; because a parent box contains its
    // children and the slab test is monotone in the box bounds, its result
    // equals a scan of the leaves in this DFS order with the per-object box
    // test, keeping the first strictly-nearer hit.
    void build_order_rec(const std::vector<int>& objs, std::vector<int>& out) const {
        size_t n = objs.size();
        if (n == 0) return;
        if (n == 1) { out.push_back(objs[0]); return; }
        auto minx = [&](int i) { return objects[i].box_lo.x; };
        if (n == 2) {
            if (minx(objs[0]) < minx(objs[1])) { out.push_back(objs[0]); out.push_back(objs[1]); }
            else { out.push_back(objs[1]); out.push_back(objs[0]); }
            return;
        }
        std::vector<size_t> idx(n);
        for (size_t i = 0; i < n; ++i) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return minx(objs[a]) < minx(objs[b]); });
        size_t mid = n / 2;
        std::vector<int> l, r;
        for (size_t i = 0; i < n; ++i) (i < mid ? l : r).push_back(objs[idx[i]]);
        build_order_rec(l, out);
        build_order_rec(r, out);
    }
    void finalize() {
        build_env_distribution();
        dfs_order.clear();
        std::vector<int> all(objects.size());
        for (size_t i = 0; i < all.size(); ++i) all[i] = (int)i;
        build_order_rec(all, dfs_order);
    }

    // TracingDetail.h:47-66 -> BoundingVolumeHierarchyDetail.h:11-101
    Hit<R> trace(const Ray<R>& ray) const {
        Hit<R> best;
        for (int id : dfs_order) {
            const Object<R>& ob = objects[id];
            if (!ref_aabb_hit(ob.box_lo, ob.box_hi, ray)) continue;
            Hit<R> g = object_hit(ob, id, ray);
            if (g.depth < best.depth) best = g;
        }
        return best;
    }
    // TracingDetail.h:68-116: trace against a single object
    Hit<R> trace_one(const Ray<R>& ray, int id) const { return object_hit(objects[id], id, ray); }
    // TracingDetail.h:118-183
    bool visible(R lightDist, const Ray<R>& ray) const {
        Hit<R> g = trace(ray);
        return g.depth > lightDist || g.depth == inf<R>();
    }
    // TracingDetail.h:185-196 (theta/phi are computed through double M_PI)
    void env_texel(const V3<R>& d, uint32_t& x, uint32_t& y) const {
        R theta = R(double(std::acos(d.y)) / M_PI);
        R phi = R((double(std::atan2(d.z, d.x)) + M_PI) / (double(2.0f) * M_PI));
        x = static_cast<uint32_t>(R(float(env_w - 1)) * phi);
        y = static_cast<uint32_t>(R(float(env_h - 1)) * theta);
        x = std::min(x, env_w - 1);
        y = std::min(y, env_h - 1);
    }
    V3<R> env_lookup(const V3<R>& d) const {
        uint32_t x, y;
        env_texel(d, x, y);
        return env[(size_t)x + (size_t)y * env_w];
    }

    // ---- albedo texture (not in the reference): a textured LAMBERT
    // object's diffuse albedo is the nearest texel of its planar projection
    // (u, v clamped to [0, 1], texel min(u * w, w - 1), min(v * h, h - 1)).
    std::vector<V3<R>> tex;
    uint32_t tex_w = 0, tex_h = 0;
    Material<R> material_at(int obj, const V3<R>& P) const {
        const Object<R>& ob = objects[obj];
        Material<R> m = ob.mat;
        if (m.type != LAMBERT || !ob.textured || tex_w == 0) return m;
        const V3<R> r = P - ob.tex_o;
        const R u = clampR(dot(r, ob.tex_u), R(0), R(1)), v = clampR(dot(r, ob.tex_v), R(0), R(1));
        const uint32_t x = std::min((uint32_t)(u * R(float(tex_w))), tex_w - 1);
        const uint32_t y = std::min((uint32_t)(v * R(float(tex_h))), tex_h - 1);
        m.albedo_d = tex[(size_t)x + (size_t)y * tex_w];
        return m;
    }

    // ---- physical estimator (not in the reference): importance sampling of
    // the environment over the cells of its nearest-texel lookup.  Cell
    // (x, y) of the cw x ch grid (cw = w-1, ch = h-1, at least 1) has texel
    // (x, y)'s value over phi in [x, x+1)/cw, theta in [y, y+1)*pi/ch; cells
    // are drawn with probability ~ mean channel value * solid angle and a
    // direction uniformly inside the cell's solid angle, so the density per
    // solid angle is the cell's mean channel value / sum(mean * solid angle).
    // Tables in float, computed in double.
    uint32_t env_cw = 0, env_ch = 0;
    std::vector<float> env_marg, env_cond, env_pdf, env_cosb;
    void build_env_distribution() {
        env_marg.clear(); env_cond.clear(); env_pdf.clear(); env_cosb.clear();
        env_cw = env_ch = 0;
        if (env_w == 0 || env_h == 0) return;
        const uint32_t cw = env_w > 1 ? env_w - 1 : 1, ch = env_h > 1 ? env_h - 1 : 1;
        env_cw = cw;
        env_ch = ch;
        const double pi = 3.14159265358979323846;
        env_cosb.resize(ch + 1);
        for (uint32_t y = 0; y <= ch; ++y) env_cosb[y] = (float)std::cos(pi * (double)y / (double)ch);
        env_cosb[0] = 1.0f;
        env_cosb[ch] = -1.0f;
        std::vector<double> lum((size_t)cw * ch), rowsum(ch), omega(ch);
        double total = 0.0;
        for (uint32_t y = 0; y < ch; ++y) {
            omega[y] = (2.0 * pi / (double)cw) * (std::cos(pi * y / (double)ch) - std::cos(pi * (y + 1) / (double)ch));
            double r = 0.0;
            for (uint32_t x = 0; x < cw; ++x) {
                const V3<R>& t = env[(size_t)x + (size_t)y * env_w];
                double l = ((double)t.x + (double)t.y + (double)t.z) / 3.0;
                if (!(l > 0.0) || !std::isfinite(l)) l = 0.0;
                lum[(size_t)y * cw + x] = l;
                r += l * omega[y];
            }
            rowsum[y] = r;
            total += r;
        }
        env_marg.resize(ch);
        env_cond.resize((size_t)cw * ch);
        env_pdf.resize((size_t)cw * ch);
        double acc = 0.0;
        for (uint32_t y = 0; y < ch; ++y) {
            acc += rowsum[y];
            env_marg[y] = total > 0.0 ? (float)(acc / total) : (float)((double)(y + 1) / (double)ch);
            double a = 0.0;
            for (uint32_t x = 0; x < cw; ++x) {
                const size_t i = (size_t)y * cw + x;
                a += lum[i] * omega[y];
                env_cond[i] = rowsum[y] > 0.0 ? (float)(a / rowsum[y]) : (float)((double)(x + 1) / (double)cw);
                env_pdf[i] = total > 0.0 ? (float)(lum[i] / total) : 0.0f;
            }
            env_cond[(size_t)y * cw + cw - 1] = 1.0f;
        }
        env_marg[ch - 1] = 1.0f;
    }
    // texel value and density per solid angle of direction d
    V3<R> env_lookup_pdf(const V3<R>& d, R& pdf) const {
        uint32_t x, y;
        env_texel(d, x, y);
        const uint32_t cx = std::min(x, env_cw - 1), cy = std::min(y, env_ch - 1);
        pdf = R(env_pdf[(size_t)cy * env_cw + cx]);
        return env[(size_t)x + (size_t)y * env_w];
    }
    static uint32_t cdf_pick(const float* c, uint32_t n, R u) {
        uint32_t lo = 0, hi = n - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (R(c[mid]) > u) hi = mid;
            else lo = mid + 1;
        }
        return lo;
    }
    // 4 draws: row, cell of the row, phi and cos(theta) inside the cell
    V3<R> env_sample(uint32_t& seed) const {
        const R u1 = rnd<R>(seed);
        const R u2 = rnd<R>(seed);
        const R u3 = rnd<R>(seed);
        const R u4 = rnd<R>(seed);
        const uint32_t y = cdf_pick(env_marg.data(), env_ch, u1);
        const uint32_t x = cdf_pick(env_cond.data() + (size_t)y * env_cw, env_cw, u2);
        const R t = (R(float(x)) + u3) / R(float(env_cw));
        const R a = R(2) * t - R(1);  // atan2(z, x) / pi
        const R sa = R(std::sin(M_PI * (double)a)), ca = R(std::cos(M_PI * (double)a));
        const R c0 = R(env_cosb[y]), c1 = R(env_cosb[y + 1]);
        const R ct = c0 - u4 * (c0 - c1);
        const R st = sqrt_(std::fmax(R(0), R(1) - ct * ct));
        return V3<R>(st * ca, ct, st * sa);
    }
};

// --------------------------------------------------------------- camera ---
// lib/include/DataStructure/Camera.h:71-75 (pose fields), Camera.cpp:6-11
template <typename R>
struct Camera { V3<R> pos, xa, ya, za; };

// TracingDetail.h:15-30 (+ KernelHelperDetail.h:13-20 index2pixel)
template <typename R> inline Ray<R> launch_ray(uint32_t px, uint32_t py, uint32_t w, uint32_t h, const Camera<R>& cam, uint32_t& seed) {
    R jx = rnd<R>(seed);
    R jy = rnd<R>(seed);
    const R rx = R(2) * ((static_cast<R>(float(px)) + jx) / R(float(w)) - R(0.5f));
    const R ry = R(2) * ((static_cast<R>(float(py)) + jy) / R(float(h)) - R(0.5f));
    V3<R> wp = cam.pos + cam.za + rx * cam.xa + ry * cam.ya;
    return Ray<R>(cam.pos, wp - cam.pos);
}

// -------------------------------------------------------- path tracing ---
// lib/src/Renderer/PathTracer.cu:97-169 (pathtracer_kernel_nee) with the
// helpers emissiveIllumintation (:20-26), directIllumination (:28-74) and
// indirectIllumination (:76-95).  Returns the path's radiance (before the
// running mean).  `stats` (optional) counts closest-hit and shadow rays.
struct RayStats { uint64_t extension = 0, shadow = 0; };

// A radiance cache that answers every query with one value: the cached path
// tracer's estimator (a non-training path ends at its first front-facing hit
// of depth >= depth that is not a mirror or glass -- beyond `depth` any
// front-facing hit, glass counting as front-facing, with `specular` -- with
// throughput * value
// in place of that vertex's emission, direct light and continuation).
template <typename R>
struct ConstantCache {
    uint32_t depth;
    V3<R> value;
    bool specular;  // mirror and glass vertices deeper than `depth` are answered too
};

template <typename R>
V3<R> trace_path(const Scene<R>& sc, const Camera<R>& cam, uint32_t tid, uint32_t w, uint32_t h,
                 uint32_t frameIndex, uint32_t maxDepth, bool rr, RayStats* stats = nullptr,
                 const ConstantCache<R>* cache = nullptr) {
    uint32_t seed = tea4(tid, frameIndex);
    uint32_t py = tid / w, px = tid - w * py;
    Ray<R> ray = launch_ray(px, py, w, h, cam, seed);
    V3<R> radiance(R(0)), rw(R(1));
    const uint32_t L = (uint32_t)sc.lights.size();
    const uint32_t useEnv = sc.env_w > 0 ? 1u : 0u;
    uint32_t depth = 0;
    do {
        bool next_valid = false;
        Hit<R> g = sc.trace(ray);
        if (stats) stats->extension++;
        if (g.depth == inf<R>()) {
            if (useEnv) radiance += rw * sc.env_lookup(ray.d);
            break;
        }
        V3<R> inc = R(-1) * ray.d;
        const Material<R> m = sc.material_at(g.obj, g.P);
        if (cache && depth >= cache->depth &&
            ((cache->specular && depth > cache->depth) ? (m.type == GLASS || dot(g.N, inc) > R(0))
                                                       : (m.type != MIRROR && m.type != GLASS && dot(g.N, inc) > R(0)))) {
            radiance += rw * cache->value;
            break;
        }
        radiance += rw * m.albedo_e;
        // directIllumination
        V3<R> N = g.N;
        if (m.type != GLASS && dot(N, inc) <= R(0)) {
            rw = V3<R>(R(0));
        } else {
            uint32_t nl = L + useEnv;
            uint32_t ls = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
            V3<R> ldir, lrad;
            R d;
            if (ls != L) {
                lrad = light_sample(sc.lights[ls], seed, g.P, ldir, d);
            } else {
                V4<R> s = sampleDirection(m, seed, inc, g.N);
                ldir = V3<R>(s.x, s.y, s.z);
                d = inf<R>();
                lrad = useEnv ? sc.env_lookup(ldir) / s.w : V3<R>(R(0));
            }
            Ray<R> shadow(g.P + R(0.001f) * ldir, ldir);
            if (stats) stats->shadow++;
            if (sc.visible(d, shadow)) {
                radiance += R(float(nl)) * std::fmax(R(0), dot(N, ldir)) * brdf(m, inc, ldir, N) * lrad * rw;
            }
        }
        if (rr) {  // PathTracer.cu:142-152
            R alpha = clampR(std::fmax(rw.x, std::fmax(rw.y, rw.z)), R(0), R(1));
            if (rnd<R>(seed) > alpha || safeFloatEqual(alpha, R(0))) break;
            rw = rw / alpha;
        }
        // indirectIllumination
        V4<R> s = sampleDirection(m, seed, inc, g.N);
        V3<R> dir(s.x, s.y, s.z);
        if (!(norm(dir) < eps<R>())) {
            rw = rw * std::abs(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
            next_valid = true;
            ray = Ray<R>(g.P + R(0.01f) * dir, dir);
        }
        if (!next_valid) break;
        ++depth;
    } while (depth < maxDepth);
    return radiance;
}

// ------------------------------------------- physical estimator (MIS) ---
// Not in the reference.  trace_path with the environment handled as a light
// that is both sampled and hit:
//   PHYS_MIS   the reference's light pick; the environment's light term
//              samples the environment (Scene::env_sample) and is weighted
//              by the power heuristic against BSDF sampling, and so is the
//              radiance of a path escaping after a non-delta bounce (camera
//              rays and delta bounces count it in full); no environment
//              light term at mirror, glass or volume-interface vertices
//   PHYS_NEE   environment light term by environment sampling at weight 1;
//              escaping paths add the environment only after a camera ray or
//              a delta bounce
//   PHYS_BSDF  lights picked among the scene's lights only; escaping paths
//              add the environment at weight 1
// All three are unbiased for the same radiance (XML lights are not
// geometry, so only the environment is reachable both ways); PHYS_MIS is
// the estimator the CUDA path implements.
enum PhysMode { PHYS_MIS = 1, PHYS_NEE = 2, PHYS_BSDF = 3 };

// density per solid angle with which sampleDirection produces `out`
template <typename R> inline R bsdf_pdf(const Material<R>& m, const V3<R>& inc, const V3<R>& out, const V3<R>& n) {
    const R c = dot(out, n);
    if (c <= R(0)) return R(0);
    if (m.type == LAMBERT || m.type == PHONG) return std::fmax(eps<R>(), c) / R(3.14159f);  // MaterialDetail.h:129
    if (m.type == GGX) {  // MaterialDetail.h:195
        const V3<R> H = normalize(inc + out);
        const R NdotH = dot(n, H);
        return D_GGX(NdotH, m.roughness) * NdotH / std::abs(R(4) * dot(inc, H));
    }
    return R(0);
}
inline bool has_delta_lobe(int type) { return type == MIRROR || type == GLASS || type == VOLUME; }
template <typename R> inline R mis_power(R a, R b) {
    const R a2 = a * a;
    return a2 / (a2 + b * b);
}

template <typename R>
V3<R> trace_path_physical(const Scene<R>& sc, const Camera<R>& cam, uint32_t tid, uint32_t w, uint32_t h,
                          uint32_t frameIndex, uint32_t maxDepth, bool rr, int mode, RayStats* stats = nullptr) {
    uint32_t seed = tea4(tid, frameIndex);
    uint32_t py = tid / w, px = tid - w * py;
    Ray<R> ray = launch_ray(px, py, w, h, cam, seed);
    V3<R> radiance(R(0)), rw(R(1));
    const uint32_t L = (uint32_t)sc.lights.size();
    const uint32_t useEnv = sc.env_w > 0 ? 1u : 0u;
    const uint32_t nl = mode == PHYS_BSDF ? L : L + useEnv;
    R last_pdf = R(0);  // BSDF density of the current ray's direction; 0: camera ray or delta bounce
    uint32_t depth = 0;
    do {
        bool next_valid = false;
        Hit<R> g = sc.trace(ray);
        if (stats) stats->extension++;
        if (g.depth == inf<R>()) {
            if (useEnv) {
                if (mode == PHYS_MIS && last_pdf > R(0)) {
                    R pe;
                    const V3<R> le = sc.env_lookup_pdf(ray.d, pe);
                    radiance += rw * (le * mis_power(last_pdf, pe / R(float(nl))));
                } else if (mode != PHYS_NEE || last_pdf == R(0)) {
                    radiance += rw * sc.env_lookup(ray.d);
                }
            }
            break;
        }
        V3<R> inc = R(-1) * ray.d;
        const Material<R> m = sc.material_at(g.obj, g.P);
        radiance += rw * m.albedo_e;
        V3<R> N = g.N;
        if (m.type != GLASS && dot(N, inc) <= R(0)) {
            rw = V3<R>(R(0));
        } else {
            uint32_t ls = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
            V3<R> ldir = N, lrad(R(0));
            R d = inf<R>();
            if (ls != L) {
                lrad = light_sample(sc.lights[ls], seed, g.P, ldir, d);
            } else if (useEnv && mode != PHYS_BSDF && !has_delta_lobe(m.type)) {
                ldir = sc.env_sample(seed);
                R pe;
                const V3<R> le = sc.env_lookup_pdf(ldir, pe);
                if (pe > R(0))
                    lrad = mode == PHYS_MIS ? le * (mis_power(pe / R(float(nl)), bsdf_pdf(m, inc, ldir, N)) / pe)
                                            : le / pe;
            }
            V3<R> contrib = R(float(nl)) * std::fmax(R(0), dot(N, ldir)) * brdf(m, inc, ldir, N) * lrad * rw;
            if (contrib.x != R(0) || contrib.y != R(0) || contrib.z != R(0)) {
                Ray<R> shadow(g.P + R(0.001f) * ldir, ldir);
                if (stats) stats->shadow++;
                if (sc.visible(d, shadow)) radiance += contrib;
            }
        }
        if (rr) {  // PathTracer.cu:142-152
            R alpha = clampR(std::fmax(rw.x, std::fmax(rw.y, rw.z)), R(0), R(1));
            if (rnd<R>(seed) > alpha || safeFloatEqual(alpha, R(0))) break;
            rw = rw / alpha;
        }
        V4<R> s = sampleDirection(m, seed, inc, g.N);
        V3<R> dir(s.x, s.y, s.z);
        if (!(norm(dir) < eps<R>())) {
            rw = rw * std::abs(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
            last_pdf = has_delta_lobe(m.type) ? R(0) : s.w;
            next_valid = true;
            ray = Ray<R>(g.P + R(0.01f) * dir, dir);
        }
        if (!next_valid) break;
        ++depth;
    } while (depth < maxDepth);
    return radiance;
}

// ------------------------------------------------------ volume tracing ---
// lib/src/Renderer/VolumeRenderer.cu:214-310 (volume_kernel) with
// handleMediumInteraction (:88-212), directIlluminationVolumetric (:24-70)
// and indirectIlluminationVolumetric (:72-86).  The reference keeps the
// current medium as a pointer into the loop-local hit record
// (`payload.volume = &(geom.material.volume)`, :276); inside an object every
// later hit is on that same object, so the medium is that object's material
// volume, and the scene volume outside.
template <typename R>
V3<R> trace_volume_path(const Scene<R>& sc, const Camera<R>& cam, uint32_t tid, uint32_t w, uint32_t h,
                        uint32_t frameIndex, uint32_t maxDepth, bool rr, RayStats* stats = nullptr,
                        bool physical = false) {
    uint32_t seed = tea4(tid, frameIndex);
    uint32_t py = tid / w, px = tid - w * py;
    Ray<R> ray = launch_ray(px, py, w, h, cam, seed);
    V3<R> radiance(R(0)), rw(R(1));
    const uint32_t L = (uint32_t)sc.lights.size();
    const uint32_t useEnv = sc.env_w > 0 ? 1u : 0u;
    const uint32_t nl = L + useEnv;
    bool inside = false;
    int obj_index = 0;
    V3<R> ray_start, out_dir;  // payload fields: persist across bounces
    uint32_t depth = 0;
    do {
        bool next_valid = false;
        Hit<R> g = inside ? sc.trace_one(ray, obj_index) : sc.trace(ray);
        if (stats) stats->extension++;
        V3<R> inc = R(-1) * ray.d;
        if (g.depth == inf<R>()) {
            if (useEnv) radiance += rw * sc.env_lookup(ray.d);
            break;
        }
        const Material<R>& m = sc.objects[g.obj].mat;
        V3<R> vss = inside ? sc.objects[obj_index].mat.sigma_s : sc.vol_sigma_s;
        V3<R> vsa = inside ? sc.objects[obj_index].mat.sigma_a : sc.vol_sigma_a;
        R vg = inside ? sc.objects[obj_index].mat.g : sc.vol_g;
        // handleMediumInteraction
        bool handled = false;
        {
            V3<R> st = vsa + vss;
            uint32_t ch = static_cast<uint32_t>(rnd<R>(seed) * R(3));
            if (!safeFloatEqual(st[ch], R(0))) {
                R t = -std::log(R(1) - rnd<R>(seed)) / st[ch];
                if (t < g.depth) {
                    handled = true;
                    V3<R> Pe = ray.o + t * ray.d;
                    R sp = vss[ch] / st[ch];
                    if (rnd<R>(seed) < sp) {
                        R pdf = 0;
                        for (int i = 0; i < 3; ++i) pdf += st[i] * std::exp(R(-1) * st[i] * t);
                        pdf /= R(3);
                        rw = rw * vss / sp * vexp(R(-1) * st * t) / pdf;
                        // medium NEE (:138-186)
                        uint32_t ls = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
                        V3<R> ldir, lrad;
                        R d;
                        if (ls != L) {
                            lrad = light_sample(sc.lights[ls], seed, Pe, ldir, d);
                        } else {
                            V4<R> s = sampleDirection(m, seed, inc, g.N);
                            ldir = V3<R>(s.x, s.y, s.z);
                            d = inf<R>();
                            lrad = useEnv ? sc.env_lookup(ldir) / s.w : V3<R>(R(0));
                        }
                        V3<R> att(R(1));
                        Ray<R> shadow(Pe + R(0.001f) * ldir, ldir);
                        if (inside) {
                            Ray<R> sray(Pe, ldir);
                            Hit<R> ge = sc.trace_one(sray, obj_index);
                            if (ge.depth == inf<R>()) { ge.depth = R(0); ge.P = Pe; }
                            att = vexp(R(-1) * st * ge.depth) * hg_phase(vg, -dot(inc, ldir));
                            shadow = Ray<R>(ge.P + R(0.001f) * ldir, ldir);
                            d -= ge.depth;
                        } else if (physical) {
                            // physical estimator: the scene medium's phase value
                            // (left out by the reference, VolumeRenderer.cu:180-186)
                            att = V3<R>(hg_phase(vg, -dot(inc, ldir)));
                        }
                        V3<R> sst = sc.vol_sigma_a + sc.vol_sigma_s;
                        if (stats) stats->shadow++;
                        if (sc.visible(d, shadow))
                            radiance += R(float(nl)) * vexp(R(-1) * sst * std::fmin(d, R(100000000.0f))) * att * lrad * rw;
                        V4<R> shg = sample_hg(vg, R(-1) * inc, seed);
                        out_dir = V3<R>(shg.x, shg.y, shg.z);
                        ray_start = Pe;
                        next_valid = true;
                    } else {
                        rw = V3<R>(R(0));  // absorbed
                    }
                } else {
                    R pdf = 0;
                    for (int i = 0; i < 3; ++i) pdf += std::exp(-st[i] * g.depth);
                    pdf /= R(3);
                    rw = rw * vexp(R(-1) * st * g.depth) / pdf;
                    ray_start = g.P;
                }
            }
        }
        if (!handled) {
            if (m.type == VOLUME) {  // medium interface (:269-278)
                V4<R> s = sampleDirection(m, seed, inc, g.N);
                out_dir = V3<R>(s.x, s.y, s.z);
                ray_start = g.P;
                bool refl = dot(inc, g.N) * dot(out_dir, g.N) > R(0);
                inside = refl ? inside : !inside;
                obj_index = g.obj;
                next_valid = true;
            } else {
                V3<R> N = g.N;
                if (m.type != GLASS && dot(N, inc) <= R(0)) {
                    rw = V3<R>(R(0));
                } else {
                    uint32_t ls = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
                    V3<R> ldir, lrad;
                    R d;
                    if (ls != L) {
                        lrad = light_sample(sc.lights[ls], seed, g.P, ldir, d);
                    } else {
                        V4<R> s = sampleDirection(m, seed, inc, g.N);
                        ldir = V3<R>(s.x, s.y, s.z);
                        d = inf<R>();
                        lrad = useEnv ? sc.env_lookup(ldir) / s.w : V3<R>(R(0));
                    }
                    Ray<R> shadow(g.P + R(0.001f) * ldir, ldir);
                    if (stats) stats->shadow++;
                    if (sc.visible(d, shadow))
                        radiance += R(float(nl)) * std::fmax(R(0), dot(N, ldir)) *
                                    vexp(R(-1) * (vss + vsa) * std::fmin(d, R(100000000.0f))) * brdf(m, inc, ldir, N) *
                                    lrad * rw;
                }
                V4<R> s = sampleDirection(m, seed, inc, g.N);
                V3<R> dir(s.x, s.y, s.z);
                if (!(norm(dir) == R(0))) {
                    rw = rw * std::abs(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
                    out_dir = dir;
                    ray_start = g.P;
                    next_valid = true;
                }
            }
            if (rr) {
                R alpha = clampR(std::fmax(rw.x, std::fmax(rw.y, rw.z)), R(0), R(1));
                if (rnd<R>(seed) > alpha || safeFloatEqual(alpha, R(0))) break;
                rw = rw / alpha;
            }
        }
        if (!next_valid) break;
        ray = Ray<R>(ray_start + R(0.001f) * out_dir, out_dir);
        ++depth;
    } while (depth < maxDepth);
    return radiance;
}

// --------------------------------------------------- gradient domain ---
// lib/src/Renderer/GradientDomain.cu: collect_radiance (:110-158) with the
// GDPT helpers (:37-108).  The base path records which vertices are valid;
// a shift path stops at the first depth whose base vertex is not valid.  The
// reference leaves never-written entries of PathData path[10] uninitialised
// (e.g. after the base path's sampled direction was rejected); they count
// as invalid here.
template <typename R>
V3<R> gdpt_collect(const Scene<R>& sc, Ray<R> ray, uint32_t seed, uint32_t maxDepth, bool shift, uint64_t& valid,
                   RayStats* stats = nullptr) {
    V3<R> radiance(R(0)), rw(R(1));
    const uint32_t L = (uint32_t)sc.lights.size();
    const uint32_t useEnv = sc.env_w > 0 ? 1u : 0u;
    const uint32_t nl = L + useEnv;
    if (!shift) valid = 0;
    uint32_t depth = 0;
    do {
        bool next_valid = false;
        if (shift && !((valid >> depth) & 1u)) return radiance;
        Hit<R> g = sc.trace(ray);
        if (stats) stats->extension++;
        if (g.depth == inf<R>()) {
            if (useEnv) radiance += rw * sc.env_lookup(ray.d);
            break;
        }
        if (!shift) valid |= (uint64_t)1 << depth;
        V3<R> inc = R(-1) * ray.d;
        const Material<R> m = sc.material_at(g.obj, g.P);
        radiance += rw * m.albedo_e;
        V3<R> N = g.N;
        if (m.type != GLASS && dot(N, inc) <= R(0)) {
            rw = V3<R>(R(0));
        } else {
            uint32_t ls = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
            V3<R> ldir, lrad;
            R d;
            if (ls != L) {
                lrad = light_sample(sc.lights[ls], seed, g.P, ldir, d);
            } else {
                V4<R> s = sampleDirection(m, seed, inc, g.N);
                ldir = V3<R>(s.x, s.y, s.z);
                d = inf<R>();
                lrad = useEnv ? sc.env_lookup(ldir) / s.w : V3<R>(R(0));
            }
            Ray<R> shadow(g.P + R(0.001f) * ldir, ldir);
            if (stats) stats->shadow++;
            if (sc.visible(d, shadow))
                radiance += R(float(nl)) * std::fmax(R(0), dot(N, ldir)) * brdf(m, inc, ldir, N) * lrad * rw;
        }
        V4<R> s = sampleDirection(m, seed, inc, g.N);
        V3<R> dir(s.x, s.y, s.z);
        if (!(norm(dir) == R(0))) {
            rw = rw * std::abs(dot(dir, g.N)) * brdf(m, inc, dir, g.N) / s.w;
            next_valid = true;
            ray = Ray<R>(g.P + R(0.01f) * dir, dir);
        }
        if (!next_valid) break;
        ++depth;
    } while (depth < maxDepth);
    return radiance;
}

// gdpt_kernel (GradientDomain.cu:160-246) for one interior pixel: base
// radiance and the forward / backward x / y gradients of this frame.
template <typename R>
void gdpt_pixel(const Scene<R>& sc, const Camera<R>& cam, uint32_t px, uint32_t py, uint32_t w, uint32_t h,
                uint32_t frameIndex, uint32_t maxDepth, V3<R> out[5], RayStats* stats = nullptr) {
    uint32_t seed = tea4(px + py * w, frameIndex);
    const int32_t off[5][2] = {{0, 0}, {-1, 0}, {1, 0}, {0, 1}, {0, -1}};  // base, left, right, up, down
    Ray<R> rays[5] = {Ray<R>(V3<R>(), V3<R>(R(0), R(0), R(1))), Ray<R>(V3<R>(), V3<R>(R(0), R(0), R(1))),
                      Ray<R>(V3<R>(), V3<R>(R(0), R(0), R(1))), Ray<R>(V3<R>(), V3<R>(R(0), R(0), R(1))),
                      Ray<R>(V3<R>(), V3<R>(R(0), R(0), R(1)))};
    uint32_t seeds[5];
    for (int k = 0; k < 5; ++k) {
        rays[k] = launch_ray((uint32_t)((int32_t)px + off[k][0]), (uint32_t)((int32_t)py + off[k][1]), w, h, cam, seed);
        seeds[k] = seed;
    }
    uint64_t valid = 0;
    V3<R> L[5];
    L[0] = gdpt_collect(sc, rays[0], seeds[0], maxDepth, false, valid, stats);
    for (int k = 1; k < 5; ++k) L[k] = gdpt_collect(sc, rays[k], seeds[k], maxDepth, true, valid, stats);
    out[0] = L[0];
    out[1] = R(0.5f) * (L[0] - L[1]);  // gradient_x_forward
    out[2] = R(0.5f) * (L[2] - L[0]);  // gradient_x_backward
    out[3] = R(0.5f) * (L[0] - L[4]);  // gradient_y_forward
    out[4] = R(0.5f) * (L[3] - L[0]);  // gradient_y_backward
}

// init_kernel (:248-273) + 50 x optimization_kernel (:303-350) with the
// device copy of temp into the output after each pass (:392-401).
// imgs: base, gxf, gxb, gyf, gyb (w*h*3 each); temp holds the reference's
// temp buffer (its border is never written); out, gx, gy receive results.
inline float gdpt_median4(const float v[4]) {  // compute_median, :275-301
    float med = 0.0f;
    uint32_t amin = 0, amax = 0;
    for (uint32_t i = 0; i < 4; ++i) {
        med += v[i];
        if (v[i] < v[amin]) amin = i;
        if (v[i] > v[amax]) amax = i;
    }
    return (med - v[amin] - v[amax]) / 2.0f;
}
inline void gdpt_reconstruct(const float* base, const float* gxf, const float* gxb, const float* gyf, const float* gyb,
                             uint32_t w, uint32_t h, float* temp, float* out, float* gx, float* gy, int iterations = 50) {
    const size_t n = (size_t)w * h;
    for (size_t p = 0; p < n; ++p) {
        uint32_t y = (uint32_t)(p / w), x = (uint32_t)(p - (size_t)w * y);
        for (int c = 0; c < 3; ++c) out[3 * p + c] = base[3 * p + c];
        if (x == 0 || y == 0 || x == w - 1 || y == h - 1) continue;
        for (int c = 0; c < 3; ++c) {
            gx[3 * p + c] = gxf[3 * p + c] + gxb[3 * p + c];
            gy[3 * p + c] = gyf[3 * p + c] + gyb[3 * p + c];
        }
    }
    for (int it = 0; it < iterations; ++it) {
        for (size_t p = 0; p < n; ++p) {
            uint32_t y = (uint32_t)(p / w), x = (uint32_t)(p - (size_t)w * y);
            if (x == 0 || y == 0 || x == w - 1 || y == h - 1) continue;
            size_t l = p - 1, r = p + 1, u = p + w, d = p - w;
            for (int c = 0; c < 3; ++c) {
                float v[4] = {out[3 * l + c] + gx[3 * l + c], out[3 * d + c] + gy[3 * d + c],
                              out[3 * r + c] - gx[3 * p + c], out[3 * u + c] - gy[3 * p + c]};
                temp[3 * p + c] = gdpt_median4(v);
            }
        }
        std::memcpy(out, temp, sizeof(float) * 3 * n);
    }
}

// raytracing_kernel (RayTracer.cu:11-54): no jitter, every light treated
// through its position and intensity, no accumulation.
template <typename R>
V3<R> raytrace_pixel(const Scene<R>& sc, const Camera<R>& cam, uint32_t tid, uint32_t w, uint32_t h) {
    uint32_t py = tid / w, px = tid - w * py;
    const R rx = R(2) * ((static_cast<R>(float(px)) + R(0)) / R(float(w)) - R(0.5f));
    const R ry = R(2) * ((static_cast<R>(float(py)) + R(0)) / R(float(h)) - R(0.5f));
    V3<R> wp = cam.pos + cam.za + rx * cam.xa + ry * cam.ya;
    Ray<R> ray(cam.pos, wp - cam.pos);
    Hit<R> g = sc.trace(ray);
    V3<R> radiance(R(0));
    if (g.depth == inf<R>()) return radiance;
    V3<R> inc = normalize(cam.pos - g.P);
    const Material<R>& m = sc.objects[g.obj].mat;
    for (const Light<R>& l : sc.lights) {
        V3<R> ldir = normalize(l.position - g.P);
        V3<R> b = brdf(m, inc, ldir, g.N);
        R d = norm(g.P - l.position);
        V3<R> lrad = l.intensity / (d * d);
        R cosTerm = std::fmax(R(0), dot(g.N, ldir));
        Ray<R> shadow(g.P - eps<R>() * ray.d, ldir);
        if (sc.visible(d, shadow)) radiance += b * lrad * cosTerm;
    }
    return radiance;
}

// PathTracer.cu:162-168 running mean
template <typename R> inline V3<R> running_mean(const V3<R>& old, const V3<R>& nw, uint32_t frameIndex) {
    if (frameIndex == 0) return nw;
    const R a = R(1) / (static_cast<R>(float(frameIndex)) + R(1));
    return (R(1) - a) * old + a * nw;
}

// ------------------------------------------------------------ tone map ---
// lib/src/Renderer/ToneMapper.cu:17-41 (REINHARD): 1 - exp() is evaluated in
// double (the literal 1.0 is a double) and the blue exponent is the double
// 1/2.2 converted to float.
inline void reinhard(const float* rgb, float exposure, uint8_t* out) {
    for (int c = 0; c < 3; ++c) {
        float e = (c == 2) ? (float)(1.0f / 2.2) : 1.0f / 2.2f;
        float m = std::pow((float)(1.0 - (double)std::exp(-rgb[c] * exposure)), e);
        out[c] = static_cast<uint8_t>(clampR(m, 0.0f, 1.0f) * 255.0f);
    }
    out[3] = 255;
}
// ToneMapper.cu:43-69 (GAMMA, sRGB OETF)
inline float srgb(float c) { return c <= 0.0031308f ? 12.92f * c : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f; }
inline void gamma(const float* rgb, uint8_t* out) {
    for (int c = 0; c < 3; ++c) out[c] = static_cast<uint8_t>(clampR(srgb(rgb[c]), 0.0f, 1.0f) * 255.0f);
    out[3] = 255;
}

// --------------------------------------------------------------- bloom ---
// lib/src/PostProcessing/PyramidConstructor.cu:9-125 driven by
// PostProcessor.cpp:125-142 with pyramid_depth 6.  The full pyramid is
// restated level by level so the oracle stays a literal check of the
// reference, including the levels whose results the output never reads.
struct ImageF { uint32_t w = 0, h = 0; std::vector<float> px; };

inline void bloom(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* out, uint32_t depth = 6) {
    std::vector<ImageF> down(depth), up(depth);
    uint32_t ww = w, hh = h;
    for (uint32_t i = 0; i < depth; ++i) {
        down[i].w = up[i].w = ww; down[i].h = up[i].h = hh;
        down[i].px.assign((size_t)ww * hh * 3, 0.0f);
        up[i].px.assign((size_t)ww * hh * 3, 0.0f);
        ww /= 2; hh /= 2;
    }
    std::memcpy(down[0].px.data(), hdr, sizeof(float) * 3 * (size_t)w * h);
    // thresholding_kernel :9-30
    for (size_t p = 0; p < (size_t)w * h; ++p) {
        float* c = &down[0].px[3 * p];
        float br = c[0] > c[1] ? c[0] : c[1];
        br = c[2] > br ? c[2] : br;
        float rq = clampR(br - th[1], 0.0f, th[2]);
        rq = th[3] * rq * rq;
        float s = std::fmax(rq, br - th[0]) / std::fmax(br, 1e-5f);
        c[0] *= s; c[1] *= s; c[2] *= s;
    }
    // downsample_kernel :32-65
    for (uint32_t d = 1; d < depth; ++d) {
        ImageF& cur = down[d];
        const ImageF& last = down[d - 1];
        for (uint32_t y = 0; y < cur.h; ++y)
            for (uint32_t x = 0; x < cur.w; ++x) {
                float r[3] = {0, 0, 0};
                const uint32_t off[4][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}};
                for (int k = 0; k < 4; ++k) {
                    uint32_t sx = 2 * x + off[k][0], sy = 2 * y + off[k][1];
                    if (sx >= last.w) sx = last.w - 1;
                    if (sy >= last.h) sy = last.h - 1;
                    const float* s = &last.px[3 * ((size_t)sx + (size_t)sy * last.w)];
                    r[0] += s[0]; r[1] += s[1]; r[2] += s[2];
                }
                float* o = &cur.px[3 * ((size_t)x + (size_t)y * cur.w)];
                o[0] = r[0] / 4.0f; o[1] = r[1] / 4.0f; o[2] = r[2] / 4.0f;
            }
    }
    up[depth - 1].px = down[depth - 1].px;
    // upscale_and_combine_kernel :67-112 (reads pyramid_down[d+1])
    const float kern[3][3] = {{1, 2, 1}, {2, 4, 2}, {1, 2, 1}};
    for (int d = (int)depth - 2; d >= 0; --d) {
        const ImageF& last = down[d + 1];
        const ImageF& cur = down[d];
        ImageF& nw = up[d];
        // A level of zero width or height (images narrower than 2^(depth-1))
        // makes the reference read outside that level; such up levels
        // (d >= 1) never reach the output, so they are skipped here.
        if (last.w == 0 || last.h == 0) continue;
        for (uint32_t y = 0; y < cur.h; ++y)
            for (uint32_t x = 0; x < cur.w; ++x) {
                float r[3] = {0, 0, 0};
                int32_t dx = (int32_t)x / 2, dy = (int32_t)y / 2;
                for (int32_t u = -1; u < 2; ++u)
                    for (int32_t v = -1; v < 2; ++v) {
                        int32_t sx = dx + u, sy = dy + v;
                        if (sx < 0) sx = 0;
                        if (sx >= (int32_t)last.w) sx = (int32_t)last.w - 1;
                        if (sy < 0) sy = 0;
                        if (sy >= (int32_t)last.h) sy = (int32_t)last.h - 1;
                        const float* s = &last.px[3 * ((size_t)sx + (size_t)sy * last.w)];
                        float k = kern[u + 1][v + 1];
                        r[0] += s[0] * k; r[1] += s[1] * k; r[2] += s[2] * k;
                    }
                size_t p = 3 * ((size_t)x + (size_t)y * cur.w);
                nw.px[p + 0] = r[0] / 16.0f + cur.px[p + 0];
                nw.px[p + 1] = r[1] / 16.0f + cur.px[p + 1];
                nw.px[p + 2] = r[2] / 16.0f + cur.px[p + 2];
            }
    }
    // combine_kernel :114-125
    for (size_t p = 0; p < 3 * (size_t)w * h; ++p) out[p] = hdr[p] + up[0].px[p];
}

// ------------------------------------------------ heterogeneous medium ---
// The density-grid medium of cupbr_b200/csrc/medium.cu, restated on the
// host.  No counterpart in the reference (VolumeRenderer.cu is homogeneous
// only), so this is checked by central differences of itself (double) and
// by the homogeneous-grid limit against the VOLUME method.  In float it
// follows the CUDA kernel's operation order, so the two agree path by path
// except where logf / sinf / cosf / powf round differently.
template <typename R>
struct Grid {
    std::vector<R> density;  // nz * ny * nx, x fastest
    uint32_t nx = 1, ny = 1, nz = 1;
    V3<R> lo, hi, inv_cell;
    R majorant = R(1), inv_majorant = R(1);
    R albedo = R(1), g = R(0), q = R(0.5f);
    R inv_q = R(2), inv_one_minus_q = R(2);  // 1 / q, 1 / (1 - q)
};

template <typename R> inline bool grid_interval(const Grid<R>& G, const V3<R>& o, const V3<R>& d, R& ta, R& tb) {
    ta = R(0);
    tb = inf<R>();
    const R os[3] = {o.x, o.y, o.z}, ds[3] = {d.x, d.y, d.z};
    const R lo[3] = {G.lo.x, G.lo.y, G.lo.z}, hi[3] = {G.hi.x, G.hi.y, G.hi.z};
    for (int a = 0; a < 3; ++a) {
        if (ds[a] == R(0)) {
            if (os[a] < lo[a] || os[a] > hi[a]) return false;
            continue;
        }
        const R inv = R(1) / ds[a];
        R t0 = (lo[a] - os[a]) * inv, t1 = (hi[a] - os[a]) * inv;
        if (t0 > t1) std::swap(t0, t1);
        ta = t0 > ta ? t0 : ta;
        tb = t1 < tb ? t1 : tb;
    }
    return ta < tb;
}

template <typename R> inline uint32_t grid_voxel(const Grid<R>& G, const V3<R>& x) {
    int ix = (int)((x.x - G.lo.x) * G.inv_cell.x);
    int iy = (int)((x.y - G.lo.y) * G.inv_cell.y);
    int iz = (int)((x.z - G.lo.z) * G.inv_cell.z);
    ix = std::min(std::max(ix, 0), (int)G.nx - 1);
    iy = std::min(std::max(iy, 0), (int)G.ny - 1);
    iz = std::min(std::max(iz, 0), (int)G.nz - 1);
    return ((uint32_t)iz * G.ny + (uint32_t)iy) * G.nx + (uint32_t)ix;
}

template <typename R> inline R grid_step(const Grid<R>& G, uint32_t& seed) {
    return -std::log(R(1) - rnd<R>(seed)) * G.inv_majorant;
}

// A light term's ratio tracking draws from its own stream, seeded from the
// path's state right after the light sample.
inline uint32_t ratio_seed(uint32_t path_seed) { return tea4(path_seed, 1u); }

// Gradient sinks of the adjoint replay.  Lrem = the sample's radiance
// minus the terms emitted so far, kept in double (as the CUDA kernels do) so
// no float cancellation residue reaches the gradients of the last vertices.
template <typename R>
struct MediumAdj {
    V3<R> delta;
    V3<double> Lrem;
    std::vector<R>* g_grid = nullptr;
    std::vector<R>* g_params = nullptr;  // [albedo, 3 per object albedo_d, 3 per object albedo_e, 3 per light]
    size_t n_objects = 0;
};

template <typename R> inline R dot_(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> inline V3<double> to_d(const V3<R>& v) { return V3<double>(double(v.x), double(v.y), double(v.z)); }
template <typename R> inline V3<R> from_d(const V3<double>& v) { return V3<R>(R(v.x), R(v.y), R(v.z)); }

// Ratio tracking over [0, len]; with adj, adds scale * dlogT/dsigma per point.
template <typename R>
R grid_ratio(const Grid<R>& G, const V3<R>& o, const V3<R>& d, R len, uint32_t& seed, std::vector<R>* g_grid,
             R scale) {
    R ta, tb;
    if (!grid_interval(G, o, d, ta, tb)) return R(1);
    tb = std::fmin(tb, len);
    R T = R(1), t = ta;
    for (int k = 0; k < (1 << 16); ++k) {
        t += grid_step(G, seed);
        if (!(t < tb)) break;
        const uint32_t v = grid_voxel(G, o + t * d);
        const R s = G.density[v];
        T *= R(1) - s * G.inv_majorant;
        if (g_grid) (*g_grid)[v] += -scale / (G.majorant - s);
    }
    return T;
}

template <typename R>
void adj_light(const Scene<R>& sc, const Grid<R>& G, MediumAdj<R>& A, const V3<R>& C, uint32_t li, const V3<R>& so,
               const V3<R>& sd, R dist, uint32_t seed_ratio, const Material<R>* m, int obj) {
    const R dc = dot_(A.delta, C);
    grid_ratio(G, so, sd, dist, seed_ratio, A.g_grid, dc);
    const Light<R>& l = sc.lights[li];
    const V3<R> Rl = l.type == 0 ? l.intensity : l.radiance;
    R* gl = A.g_params->data() + 1 + 6 * A.n_objects + 3 * li;
    if (Rl.x != R(0)) gl[0] += A.delta.x * C.x / Rl.x;
    if (Rl.y != R(0)) gl[1] += A.delta.y * C.y / Rl.y;
    if (Rl.z != R(0)) gl[2] += A.delta.z * C.z / Rl.z;
    if (m && m->type == LAMBERT) {
        R* ga = A.g_params->data() + 1 + 3 * (size_t)obj;
        if (m->albedo_d.x != R(0)) ga[0] += A.delta.x * C.x / m->albedo_d.x;
        if (m->albedo_d.y != R(0)) ga[1] += A.delta.y * C.y / m->albedo_d.y;
        if (m->albedo_d.z != R(0)) ga[2] += A.delta.z * C.z / m->albedo_d.z;
    }
    A.Lrem = A.Lrem - to_d(C);
}

// One sample of the grid-medium estimator (A == nullptr: forward only;
// Lsum, if given, receives the terms' sum in double).
template <typename R>
V3<R> medium_path(const Scene<R>& sc, const Grid<R>& G, Ray<R> ray, uint32_t seed, uint32_t maxDepth,
                  MediumAdj<R>* A, V3<double>* Lsum = nullptr) {
    V3<R> L(R(0)), beta(R(1));
    const uint32_t nl = (uint32_t)sc.lights.size();
    for (uint32_t depth = 0; depth < maxDepth; ++depth) {
        Hit<R> hit = sc.trace(ray);
        bool scatter = false;
        V3<R> x;
        R ta, tb;
        if (grid_interval(G, ray.o, ray.d, ta, tb)) {
            tb = std::fmin(tb, hit.depth);
            R t = ta;
            for (int k = 0;; ++k) {
                if (k == (1 << 16)) return L;
                t += grid_step(G, seed);
                if (!(t < tb)) break;
                const V3<R> xp = ray.o + t * ray.d;
                const uint32_t v = grid_voxel(G, xp);
                const R s = G.density[v];
                const R xi = rnd<R>(seed);
                bool real;
                if (G.q <= R(0)) {
                    real = xi < s * G.inv_majorant;
                    if (real) {
                        beta = G.albedo * beta;
                        if (A) (*A->g_params)[0] += dot_(A->delta, from_d<R>(A->Lrem)) / G.albedo;
                    }
                } else {
                    real = s > R(0) && xi < G.q;
                    if (real) {
                        beta = (G.albedo * s * G.inv_majorant * G.inv_q) * beta;
                        if (A) {
                            const R lr = dot_(A->delta, from_d<R>(A->Lrem));
                            (*A->g_grid)[v] += lr / s;
                            (*A->g_params)[0] += lr / G.albedo;
                        }
                    } else if (s > R(0)) {
                        beta = ((R(1) - s * G.inv_majorant) * G.inv_one_minus_q) * beta;
                        if (A) (*A->g_grid)[v] += -dot_(A->delta, from_d<R>(A->Lrem)) / (G.majorant - s);
                    }
                }
                if (real) {
                    scatter = true;
                    x = xp;
                    break;
                }
            }
        }
        if (scatter) {
            if (nl > 0) {
                const uint32_t li = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
                V3<R> ldir;
                R dist;
                const V3<R> lrad = light_sample(sc.lights[li], seed, x, ldir, dist);
                const Ray<R> sh(x, ldir);
                const uint32_t seed_ratio = ratio_seed(seed);
                uint32_t sr = seed_ratio;
                const R T = grid_ratio(G, sh.o, sh.d, dist, sr, (std::vector<R>*)nullptr, R(0));
                if (sc.visible(dist, sh)) {
                    const V3<R> C = T * ((R(float(nl)) * hg_phase(G.g, dot(ray.d, sh.d))) * (lrad * beta));
                    L += C;
                    if (Lsum) *Lsum += to_d(C);
                    if (A) adj_light(sc, G, *A, C, li, sh.o, sh.d, dist, seed_ratio, (const Material<R>*)nullptr, 0);
                }
            }
            const V4<R> sp = sample_hg(G.g, ray.d, seed);
            ray = Ray<R>(x, V3<R>(sp.x, sp.y, sp.z));
            continue;
        }
        if (hit.depth == inf<R>()) break;
        const Material<R>& m = sc.objects[hit.obj].mat;
        const V3<R> inc = R(-1) * ray.d;
        const V3<R> N = hit.N;
        const V3<R> Ce = beta * m.albedo_e;
        if (A) {  // dL/dalbedo_e = the path weight at this hit
            R* ge = A->g_params->data() + 1 + 3 * A->n_objects + 3 * (size_t)hit.obj;
            ge[0] += A->delta.x * beta.x;
            ge[1] += A->delta.y * beta.y;
            ge[2] += A->delta.z * beta.z;
        }
        L += Ce;
        if (Lsum) *Lsum += to_d(Ce);
        if (A) A->Lrem = A->Lrem - to_d(Ce);
        if (m.type != GLASS && dot(N, inc) <= R(0)) break;
        if (nl > 0) {
            const uint32_t li = static_cast<uint32_t>(rnd<R>(seed) * R(float(nl)));
            V3<R> ldir;
            R dist;
            const V3<R> lrad = light_sample(sc.lights[li], seed, hit.P, ldir, dist);
            const Ray<R> sh(hit.P + R(0.001f) * ldir, ldir);
            const uint32_t seed_ratio = ratio_seed(seed);
            uint32_t sr = seed_ratio;
            const R T = grid_ratio(G, sh.o, sh.d, dist, sr, (std::vector<R>*)nullptr, R(0));
            if (sc.visible(dist, sh)) {
                const V3<R> C =
                    T * ((R(float(nl)) * std::fmax(R(0), dot(N, ldir))) * (brdf(m, inc, ldir, N) * lrad * beta));
                L += C;
                if (Lsum) *Lsum += to_d(C);
                if (A) adj_light(sc, G, *A, C, li, sh.o, sh.d, dist, seed_ratio, &m, hit.obj);
            }
        }
        const V4<R> sp = sampleDirection(m, seed, inc, N);
        const V3<R> dir(sp.x, sp.y, sp.z);
        if (norm(dir) < eps<R>()) break;
        beta = beta * std::abs(dot(dir, N)) * brdf(m, inc, dir, N) / sp.w;
        if (A && m.type == LAMBERT) {
            R* ga = A->g_params->data() + 1 + 3 * (size_t)hit.obj;
            const V3<R> lr = from_d<R>(A->Lrem);
            if (m.albedo_d.x != R(0)) ga[0] += A->delta.x * lr.x / m.albedo_d.x;
            if (m.albedo_d.y != R(0)) ga[1] += A->delta.y * lr.y / m.albedo_d.y;
            if (m.albedo_d.z != R(0)) ga[2] += A->delta.z * lr.z / m.albedo_d.z;
        }
        if (beta.x == R(0) && beta.y == R(0) && beta.z == R(0)) break;
        ray = Ray<R>(hit.P + R(0.01f) * dir, dir);
    }
    return L;
}

// Pixel tid: mean over samples frame0 .. frame0 + spp - 1.
template <typename R>
V3<R> medium_pixel(const Scene<R>& sc, const Grid<R>& G, const Camera<R>& cam, uint32_t tid, uint32_t w, uint32_t h,
                   uint32_t spp, uint32_t frame0, uint32_t maxDepth) {
    V3<R> acc(R(0));
    for (uint32_t s = 0; s < spp; ++s) {
        uint32_t seed = tea4(tid, frame0 + s);
        const uint32_t py = tid / w, px = tid - w * py;
        const Ray<R> ray = launch_ray(px, py, w, h, cam, seed);
        acc += medium_path(sc, G, ray, seed, maxDepth, (MediumAdj<R>*)nullptr);
    }
    return acc / R(float(spp));
}

// Adds pixel tid's share of dLoss/dtheta for dLoss/dI = grad (RGB).
template <typename R>
void medium_pixel_adjoint(const Scene<R>& sc, const Grid<R>& G, const Camera<R>& cam, uint32_t tid, uint32_t w,
                          uint32_t h, uint32_t spp, uint32_t frame0, uint32_t maxDepth, const V3<R>& grad,
                          std::vector<R>& g_grid, std::vector<R>& g_params) {
    MediumAdj<R> A;
    A.delta = grad / R(float(spp));
    if (A.delta.x == R(0) && A.delta.y == R(0) && A.delta.z == R(0)) return;
    A.g_grid = &g_grid;
    A.g_params = &g_params;
    A.n_objects = sc.objects.size();
    for (uint32_t s = 0; s < spp; ++s) {
        uint32_t seed = tea4(tid, frame0 + s);
        const uint32_t py = tid / w, px = tid - w * py;
        const Ray<R> ray = launch_ray(px, py, w, h, cam, seed);
        V3<double> Ls(0.0);
        medium_path(sc, G, ray, seed, maxDepth, (MediumAdj<R>*)nullptr, &Ls);
        A.Lrem = Ls;
        medium_path(sc, G, ray, seed, maxDepth, &A);
    }
}

}  // namespace oracle
