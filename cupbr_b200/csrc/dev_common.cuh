// Device-side types and arithmetic shared by the cupbr-b200 kernels.
//
// Translation units that include this header are compiled with -fmad=false
// and IEEE division / square root (no -use_fast_math): every +,-,*,/ and
// sqrt below is a single correctly rounded operation in the reference's
// operation order, so hit distances, camera rays and BSDF algebra equal the
// reference's __host__ __device__ code run on the CPU bit for bit; only the
// transcendental functions (cosf, sinf, expf, powf, acosf, atan2f) may differ
// in the last place.  Where a fused multiply-add is wanted (the BVH box
// test) it is written out with __fmaf_rn.
#pragma once

#include <cstdint>
#include <math.h>
#include <cuda_runtime.h>

namespace cupbr_b200 {

#define CUPBR_EPS 1e-5f  // lib/include/Math/Functions.h:4
#define CUPBR_PIF 3.14159265358979323846f

struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ f3 splat(float v) { return {v, v, v}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// scalar * vector (VectorOperationsDetail.h:112-116); vector * scalar forwards here
__host__ __device__ __forceinline__ f3 operator*(float s, f3 v) { return {s * v.x, s * v.y, s * v.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 v, float s) { return {s * v.x, s * v.y, s * v.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 v, float s) { return {v.x / s, v.y / s, v.z / s}; }
__host__ __device__ __forceinline__ void operator+=(f3& a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
__host__ __device__ __forceinline__ float dot(f3 v, f3 w) { return v.x * w.x + v.y * w.y + v.z * w.z; }
__host__ __device__ __forceinline__ f3 cross(f3 v, f3 w) {
    return {v.y * w.z - v.z * w.y, v.z * w.x - v.x * w.z, v.x * w.y - v.y * w.x};
}
__host__ __device__ __forceinline__ float norm(f3 v) { return sqrtf(dot(v, v)); }
__host__ __device__ __forceinline__ f3 normalize(f3 v) { return v / norm(v); }
__host__ __device__ __forceinline__ bool is_zero(f3 v) { return v.x == 0.0f && v.y == 0.0f && v.z == 0.0f; }

__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float4 f4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// ------------------------------------------------------------- RNG ---
// lib/src/Math/FunctionsDetail.h:70-87
__host__ __device__ __forceinline__ uint32_t tea4(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
// FunctionsDetail.h:89-98
__host__ __device__ __forceinline__ float rnd(uint32_t& s) {
    s = 1664525u * s + 1013904223u;
    return (float)(s & 0x00FFFFFFu) / (float)0x01000000;
}

// ------------------------------------------------------------ math ---
// FunctionsDetail.h:10-15, 24-29
__device__ __forceinline__ bool feq0(float v) { return fabsf(v) < CUPBR_EPS; }
__device__ __forceinline__ float delta(float v) { return feq0(v) ? 1.0f : 0.0f; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
// FunctionsDetail.h:31-36
__device__ __forceinline__ f3 reflect(f3 inc, f3 n) { return normalize((2.0f * dot(inc, n)) * n - inc); }
// FunctionsDetail.h:38-52
__device__ __forceinline__ f3 refract(float eta, f3 inc, f3 n) {
    float NdotI = dot(inc, n);
    float k = 1.0f - eta * eta * (1.0f - NdotI * NdotI);
    if (k < 0.0f) return splat(0.0f);
    return (-eta) * inc - ((-eta) * NdotI + sqrtf(k)) * n;
}
// FunctionsDetail.h:54-68
__device__ __forceinline__ float fresnel(float F0, float VdotH) {
    float p = fmaxf(0.0f, 1.0f - VdotH);
    return F0 + (1.0f - F0) * p * p * p * p * p;
}
__device__ __forceinline__ f3 fresnel3(f3 F0, float VdotH) {
    float p = fmaxf(0.0f, 1.0f - VdotH);
    return F0 + (splat(1.0f) - F0) * p * p * p * p * p;
}
// FunctionsDetail.h:100-117
__device__ __forceinline__ f3 to_local_frame(f3 N, f3 d) {
    const float x = N.x, y = N.y, z = N.z;
    const float sz = (z >= 0.0f) ? 1.0f : -1.0f;
    const float a = 1.0f / (sz + z);
    const float ya = y * a;
    const float b = x * ya;
    const float c = x * sz;
    f3 lx = mk(c * x * a - 1.0f, sz * b, c);
    f3 ly = mk(b, y * ya - sz, y);
    return d.x * lx + d.y * ly + d.z * N;
}

// ------------------------------------------------------- scene data ---
// Material as uploaded (Material.h:34-42); brdf_lambert's albedo_d/pi is
// precomputed on the host with the same single IEEE division.
struct DMaterial {
    float4 e;   // albedo_e.xyz, type (as float)
    float4 d;   // albedo_d.xyz, shininess
    float4 s;   // albedo_s.xyz, roughness
    float4 dl;  // albedo_d / (float)M_PI, eta
    float4 ss;  // sigma_s.xyz, g
    float4 sa;  // sigma_a.xyz, interface (1 = GLASS)
};

// Per-object record: the reference's object box (finite for SPHERE / MESH,
// infinite otherwise) feeds the reference's per-object slab test.
struct DObject {
    float4 lo;  // box lo.xyz, finite flag
    float4 hi;  // box hi.xyz, material index (as int bits)
};

struct DLight {  // Light.h:20-71 with the area light's normal and area precomputed
    float4 pos;  // position.xyz, type
    float4 I;    // intensity.xyz
    float4 L;    // radiance.xyz, area
    float4 e1;   // halfExtend1
    float4 e2;   // halfExtend2
    float4 n;    // normalize(cross(e1, e2))
};

struct DeviceScene {
    const float4* __restrict__ nodes;     // 4 per node
    const float4* __restrict__ tris;      // 3 per triangle slot: (v1, key), (v2 - v1, obj), (v3 - v1, 0)
    const float4* __restrict__ tri_n;     // 1 per triangle slot: normal.xyz
    const float4* __restrict__ spheres;   // 2 per sphere slot: (center, key), (radius, radius^2, obj, 0)
    const float4* __restrict__ quads;     // 4 per quad slot: (pos, key), (n, PdotN), (e1, |e1|^2), (e2, |e2|^2)
    const int32_t* __restrict__ quad_obj; // object id per quad slot
    const float4* __restrict__ planes;    // 2 per plane: (pos, key), (n, obj)
    const DObject* __restrict__ objects;
    const DMaterial* __restrict__ materials;
    const DLight* __restrict__ lights;
    const float4* __restrict__ env;       // env_w * env_h RGB (w unused)
    const int4* __restrict__ obj_info;    // per object: (geometry type, first key, primitive count, 0)
    const uint32_t* __restrict__ key_slot; // per primitive key: slot in its type's table (planes: plane index)
    uint32_t n_nodes, n_tris, n_spheres, n_quads, n_planes, n_objects, n_lights;
    uint32_t env_w, env_h;
    // environment importance sampling (env_dist.hpp): env_ch row CDF, env_ch x
    // env_cw cell CDFs and densities per solid angle, env_ch + 1 row-boundary cosines
    const float* __restrict__ env_marg;
    const float* __restrict__ env_cond;
    const float* __restrict__ env_pdf;
    const float* __restrict__ env_cosb;
    uint32_t env_cw, env_ch;
    // albedo texture (tex_w * tex_h texels, RGB in xyz) and per object its
    // planar projection: (origin, textured flag), (u axis / |u|^2, 0),
    // (v axis / |v|^2, 0); null without a texture
    float4* tex;
    const float4* __restrict__ obj_tex;
    uint32_t tex_w, tex_h;
    uint32_t sphere_base, quad_base;      // unified slot offsets (triangles start at 0)
    float4 vol_sigma_s, vol_sigma_a;      // scene medium (Scene.h:23), w = g in sigma_s
};

// Hit record written by the closest-hit pass: t and the primitive ref
// (type in bits 30..31: 0 triangle, 1 sphere, 2 quad, 3 plane; slot below).
constexpr int32_t HIT_NONE = -1;
__host__ __device__ __forceinline__ int32_t prim_ref(int type, uint32_t slot) { return (int32_t)(((uint32_t)type << 30) | slot); }
__host__ __device__ __forceinline__ int prim_type(int32_t r) { return (int)((uint32_t)r >> 30); }
__host__ __device__ __forceinline__ uint32_t prim_slot(int32_t r) { return (uint32_t)r & 0x3FFFFFFFu; }

}  // namespace cupbr_b200
