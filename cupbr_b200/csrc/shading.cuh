// BSDF sampling / evaluation, light sampling and the environment lookup in
// the reference's arithmetic order (MaterialDetail.h, LightDetail.h,
// TracingDetail.h:185-196).  See dev_common.cuh for the rounding contract.
#pragma once

#include "dev_common.cuh"

namespace cupbr_b200 {

struct MatView {
    int type;
    f3 albedo_e, albedo_d, albedo_s, albedo_d_over_pi;
    float shininess, roughness, eta;
    f3 sigma_s, sigma_a;
    float g;
    bool interface_glass;
};

__device__ __forceinline__ MatView load_material(const DMaterial* __restrict__ mats, int idx) {
    const DMaterial* m = mats + idx;
    float4 e = __ldg(&m->e), d = __ldg(&m->d), s = __ldg(&m->s), dl = __ldg(&m->dl);
    MatView v;
    v.type = (int)e.w;
    v.albedo_e = xyz(e);
    v.albedo_d = xyz(d);
    v.shininess = d.w;
    v.albedo_s = xyz(s);
    v.roughness = s.w;
    v.albedo_d_over_pi = xyz(dl);
    v.eta = dl.w;
    float4 ss = __ldg(&m->ss), sa = __ldg(&m->sa);
    v.sigma_s = xyz(ss);
    v.g = ss.w;
    v.sigma_a = xyz(sa);
    v.interface_glass = sa.w != 0.0f;
    return v;
}

// MaterialDetail.h:13-31
__device__ __forceinline__ float d_ggx(float NdotH, float roughness) {
    float a2 = roughness * roughness;
    float d = (NdotH * a2 - NdotH) * NdotH + 1.0f;
    return a2 / ((float)3.14159265358979323846 * d * d);
}
__device__ __forceinline__ float v_smith_joint_ggx(float NdotL, float NdotV, float roughness) {
    float a2 = roughness * roughness;
    float denomA = NdotV * sqrtf(a2 + (1.0f - a2) * NdotL * NdotL);
    float denomB = NdotL * sqrtf(a2 + (1.0f - a2) * NdotV * NdotV);
    float G = 2.0f * NdotL * NdotV / (denomA + denomB + CUPBR_EPS);
    return G / (4.0f * NdotV * NdotL + CUPBR_EPS);
}

// MaterialDetail.h:217-223
__device__ __forceinline__ f3 brdf_mirror(const MatView& m, f3 inc, f3 out, f3 n) {
    f3 r = reflect(inc, n);
    return m.albedo_s * delta(1.0f - dot(out, r)) / dot(out, n);
}

// MaterialDetail.h:35-74 with the per-type bodies of :202-274
__device__ __forceinline__ f3 brdf(const MatView& m, f3 inc, f3 out, f3 n) {
    switch (m.type) {
        case 0: return m.albedo_d_over_pi;
        case 1: {
            f3 h = normalize(inc + out);
            return m.albedo_s * powf(fmaxf(0.0f, dot(h, n)), m.shininess) + m.albedo_d_over_pi;
        }
        case 2: return brdf_mirror(m, inc, out, n);
        case 3: {
            if (dot(inc, n) * dot(out, n) > 0.0f) {
                if (dot(inc, n) > 0.0f) return brdf_mirror(m, inc, out, n);
                return brdf_mirror(m, inc, out, -1.0f * n);
            }
            f3 refracted, nn = n;
            if (dot(inc, n) > 0.0f) {
                refracted = refract(1.0f / m.eta, inc, n);
            } else {
                refracted = refract(m.eta, inc, -1.0f * n);
                nn = -1.0f * n;
            }
            return m.albedo_s * delta(1.0f - dot(refracted, out)) / dot(inc, nn);
        }
        case 4: {
            f3 H = normalize(inc + out);
            float NdotH = dot(n, H), LdotH = dot(out, H), NdotL = dot(n, out), NdotV = dot(n, inc);
            float ndf = d_ggx(NdotH, m.roughness);
            float vis = v_smith_joint_ggx(NdotL, NdotV, m.roughness);
            return ndf * vis * fresnel3(m.albedo_s, LdotH);
        }
        default: return splat(0.0f);
    }
}

// MaterialDetail.h:143-169
__device__ __forceinline__ float4 sample_glass(const MatView& m, uint32_t& seed, f3 inc, f3 n0) {
    const float NdotV = dot(inc, n0);
    bool outside = NdotV > 0.0f;
    float e = outside ? 1.0f / m.eta : m.eta;
    f3 n = outside ? n0 : -1.0f * n0;
    float F0 = (m.eta - 1.0f) / (m.eta + 1.0f);
    F0 *= F0;
    float p_reflect = fresnel(F0, fabsf(dot(inc, n)));
    float xi = rnd(seed);
    f3 refr = refract(e, inc, n);
    f3 d;
    if (xi <= p_reflect || feq0(norm(refr))) d = reflect(inc, n);
    else d = normalize(refr);
    return f4(d, 1.0f);
}

// MaterialDetail.h:76-200
__device__ __forceinline__ float4 sample_direction(const MatView& m, uint32_t& seed, f3 inc, f3 n) {
    switch (m.type) {
        case 0:
        case 1: {  // :113-132
            const float xi1 = rnd(seed);
            const float xi2 = rnd(seed);
            const float r = sqrtf(xi1);
            const float phi = (2.0f * 3.14159f) * xi2;
            float s, c;
            sincosf(phi, &s, &c);
            const float x = r * c;
            const float y = r * s;
            const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
            f3 d = normalize(to_local_frame(n, mk(x, y, z)));
            float p = fmaxf(CUPBR_EPS, dot(d, n)) / 3.14159f;
            return f4(d, p);
        }
        case 2: return f4(reflect(inc, n), 1.0f);  // :134-141
        case 3: return sample_glass(m, seed, inc, n);
        case 4: {  // :171-200
            float u = rnd(seed);
            float v = rnd(seed);
            float cosTheta = sqrtf((1.0f - u) / (1.0f + (m.roughness * m.roughness - 1.0f) * u));
            float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
            float phi = (2.0f * (float)3.14159265358979323846) * v;
            float s, c;
            sincosf(phi, &s, &c);
            float x = sinTheta * c;
            float y = sinTheta * s;
            float z = cosTheta;
            f3 H = to_local_frame(n, mk(x, y, z));
            f3 L = reflect(inc, H);
            float LdotH = dot(inc, H);
            float NdotH = dot(n, H);
            if (dot(n, L) <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            float p = d_ggx(NdotH, m.roughness) * NdotH / fabsf(4.0f * LdotH);
            return f4(L, p);
        }
        case 5:
            return m.interface_glass ? sample_glass(m, seed, inc, n) : f4(-1.0f * inc, 1.0f);
    }
    return make_float4(__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000),
                       __int_as_float(0x7f800000));
}

// MaterialDetail.h:276-313 (Henyey-Greenstein)
__device__ __forceinline__ float hg_phase(float g, float cos_theta) {
    if (fabsf(g) < 1e-3f) return (float)(0.25 / (double)(float)3.14159265358979323846);
    float g2 = g * g;
    float area = 4.0f * 3.14159f;
    return (1.0f - g2) / area * powf(1.0f + g2 - 2.0f * g * cos_theta, -1.5f);
}
__device__ __forceinline__ float4 sample_hg(float g_, f3 forward, uint32_t& seed) {
    float g = g_ < 0.0f ? fminf((float)-1e-3, g_) : fmaxf((float)1e-3, g_);
    float u1 = rnd(seed);
    float u2 = rnd(seed);
    float g2 = g * g;
    float d = (1.0f - g2) / (1.0f - g + 2.0f * g * u1);
    float cos_theta = clampf(0.5f / g * (1.0f + g2 - d * d), -1.0f, 1.0f);
    float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
    float phi = (2.0f * 3.14159f) * u2;
    float s, c;
    sincosf(phi, &s, &c);
    f3 res = normalize(to_local_frame(forward, mk(sin_theta * c, sin_theta * s, cos_theta)));
    return f4(res, hg_phase(g, dot(forward, res)));
}

// LightDetail.h:8-52 (area normal and area precomputed in DLight)
__device__ __forceinline__ f3 sample_light(const DLight* __restrict__ lights, uint32_t idx, uint32_t& seed, f3 P, f3& dir,
                                           float& dist) {
    const DLight* l = lights + idx;
    float4 pos = __ldg(&l->pos);
    if (pos.w == 0.0f) {  // POINT
        f3 lp = xyz(pos);
        dir = normalize(lp - P);
        dist = norm(lp - P);
        return xyz(__ldg(&l->I)) / (dist * dist);
    }
    float xi1 = rnd(seed) * 2.0f - 1.0f;
    float xi2 = rnd(seed) * 2.0f - 1.0f;
    float4 L = __ldg(&l->L);
    f3 s = xyz(pos) + xi1 * xyz(__ldg(&l->e1)) + xi2 * xyz(__ldg(&l->e2));
    f3 n = xyz(__ldg(&l->n));
    dir = normalize(s - P);
    dist = norm(s - P);
    float NdotL = dot(dir, n);
    if (NdotL < 0.0f) NdotL *= -1.0f;
    float solidAngle = L.w * NdotL / (dist * dist);
    return xyz(L) * solidAngle;
}

// TracingDetail.h:185-196: theta and phi go through the double M_PI
__device__ __forceinline__ void env_texel(const DeviceScene& S, f3 d, uint32_t& x, uint32_t& y) {
    const double PI_D = 3.14159265358979323846;
    float theta = (float)((double)acosf(d.y) / PI_D);
    float phi = (float)(((double)atan2f(d.z, d.x) + PI_D) / ((double)2.0f * PI_D));
    x = (uint32_t)((float)(S.env_w - 1) * phi);
    y = (uint32_t)((float)(S.env_h - 1) * theta);
    x = min(x, S.env_w - 1);
    y = min(y, S.env_h - 1);
}
__device__ __forceinline__ f3 env_lookup(const DeviceScene& S, f3 d) {
    uint32_t x, y;
    env_texel(S, d, x, y);
    return xyz(__ldg(&S.env[(size_t)x + (size_t)y * S.env_w]));
}

// Albedo texture (no counterpart in the reference): the texel a textured
// object's planar projection puts point P on, or -1 (no texture, object not
// textured); `a` receives the texel's RGB.
__device__ __forceinline__ int32_t tex_lookup(const DeviceScene& S, int32_t obj, f3 P, f3& a) {
    if (!S.obj_tex) return -1;
    const float4 o = __ldg(&S.obj_tex[3 * (size_t)obj]);
    if (o.w == 0.0f) return -1;
    const f3 r = P - xyz(o);
    const float u = clampf(dot(r, xyz(__ldg(&S.obj_tex[3 * (size_t)obj + 1]))), 0.0f, 1.0f);
    const float v = clampf(dot(r, xyz(__ldg(&S.obj_tex[3 * (size_t)obj + 2]))), 0.0f, 1.0f);
    const uint32_t x = min((uint32_t)(u * (float)S.tex_w), S.tex_w - 1);
    const uint32_t y = min((uint32_t)(v * (float)S.tex_h), S.tex_h - 1);
    const int32_t t = (int32_t)(x + y * S.tex_w);
    a = xyz(S.tex[t]);
    return t;
}

// ------------------------------------------------ physical estimator (MIS) ---
// Not in the reference (its estimator is restated above and stays the
// default): environment importance sampling over the lookup's cells
// (env_dist.hpp) combined with BSDF sampling by the power heuristic.

// Texel value and density per solid angle of the environment in direction d.
__device__ __forceinline__ f3 env_lookup_pdf(const DeviceScene& S, f3 d, float& pdf) {
    uint32_t x, y;
    env_texel(S, d, x, y);
    const uint32_t cx = min(x, S.env_cw - 1), cy = min(y, S.env_ch - 1);
    pdf = __ldg(&S.env_pdf[(size_t)cy * S.env_cw + cx]);
    return xyz(__ldg(&S.env[(size_t)x + (size_t)y * S.env_w]));
}
// First index of the n ascending entries of c above u (n - 1 if none).
__device__ __forceinline__ uint32_t cdf_pick(const float* __restrict__ c, uint32_t n, float u) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&c[mid]) > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}
// A direction drawn from the environment's distribution (4 draws): a row by
// its CDF, a cell of the row by the row's CDF, then uniform over the cell's
// solid angle (phi uniform, cos(theta) uniform between the row's bounds).
__device__ __forceinline__ f3 env_sample(const DeviceScene& S, uint32_t& seed) {
    const float u1 = rnd(seed);
    const float u2 = rnd(seed);
    const float u3 = rnd(seed);
    const float u4 = rnd(seed);
    const uint32_t y = cdf_pick(S.env_marg, S.env_ch, u1);
    const uint32_t x = cdf_pick(S.env_cond + (size_t)y * S.env_cw, S.env_cw, u2);
    const float t = ((float)x + u3) / (float)S.env_cw;  // phi in [0, 1]
    float sa, ca;
    sincospif(2.0f * t - 1.0f, &sa, &ca);             // atan2(z, x) = 2 pi phi - pi
    const float c0 = __ldg(&S.env_cosb[y]), c1 = __ldg(&S.env_cosb[y + 1]);
    const float ct = c0 - u4 * (c0 - c1);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    return mk(st * ca, ct, st * sa);
}
// Density per solid angle with which sample_direction produces `out`
// (0 for the delta lobes of mirror, glass and the volume interface).
__device__ __forceinline__ float bsdf_pdf(const MatView& m, f3 inc, f3 out, f3 n) {
    const float c = dot(out, n);
    if (c <= 0.0f) return 0.0f;
    if (m.type == 0 || m.type == 1) return fmaxf(CUPBR_EPS, c) / 3.14159f;  // MaterialDetail.h:129
    if (m.type == 4) {                                                     // MaterialDetail.h:195
        const f3 H = normalize(inc + out);
        const float NdotH = dot(n, H);
        return d_ggx(NdotH, m.roughness) * NdotH / fabsf(4.0f * dot(inc, H));
    }
    return 0.0f;
}
__device__ __forceinline__ bool has_delta_lobe(int type) { return type == 2 || type == 3 || type == 5; }
// Power heuristic weight of technique a against b.
__device__ __forceinline__ float mis_power(float a, float b) {
    const float a2 = a * a;
    return a2 / (a2 + b * b);
}

}  // namespace cupbr_b200
