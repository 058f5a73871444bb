// Host build of the REFERENCE's own code (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/build_oracle.py with g++ against the reference sources
// where they lie (lib/include, lib/src) into oracle/_ref/libref_host.so.  It
// builds a cupbr::Scene with the reference's own classes -- Plane, Sphere,
// Quad, Triangle, Mesh constructors, Light, Material, Image and the object
// BVH constructor (BoundingVolumeHierarchy.cpp:46-136, whose cudaMalloc /
// cudaMemcpy calls land in oracle/cuda_host_shim.cpp) -- and then calls the
// reference's __host__ __device__ functions on the CPU:
//   Tracing::traceRay / traceVisibility / launchRay / direction2UV
//   (TracingDetail.h), BoundingVolumeHierarchy::computeRayIntersection,
//   Material::brdf / sampleDirection, Light::sample, Math::tea / rnd.
// Only the body of the __global__ kernel pathtracer_kernel_nee
// (PathTracer.cu:97-169) and its three __device__ helpers (:20-95), which
// live in a .cu file that also holds a <<<>>> launch, are written out here in
// the same statement order.  The outputs are the golden vectors under
// tests/golden/ that pin the oracle (oracle/oracle.hpp).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

#include <Core/Tracing.h>
#include <DataStructure/BoundingVolumeHierarchy.h>
#include <DataStructure/Camera.h>
#include <DataStructure/Light.h>
#include <Geometry/Material.h>
#include <Scene/Scene.h>

using namespace cupbr;

namespace {

struct RefScene {
    Scene scene;
    std::vector<Geometry*> geometry;
    std::vector<Light*> lights;
    std::vector<Vector3float> env;
    BoundingVolumeHierarchy* bvh = nullptr;
};

Vector3float v3(const float* p) { return Vector3float(p[0], p[1], p[2]); }

Material material_of(const float* m) {
    Material mat;
    mat.type = static_cast<MaterialType>((int)m[0]);
    mat.albedo_e = v3(m + 1);
    mat.albedo_d = v3(m + 4);
    mat.albedo_s = v3(m + 7);
    mat.shininess = m[10];
    mat.roughness = m[11];
    mat.eta = m[12];
    mat.volume.sigma_s = v3(m + 13);
    mat.volume.sigma_a = v3(m + 16);
    mat.volume.g = m[19];
    mat.volume.interface = m[20] != 0.0f ? Interface::GLASS : Interface::NONE;
    return mat;
}

// Camera pose fields are private (Camera.h:71-75) and the class is standard
// layout: the first four Vector3float members are overwritten in place.
Camera camera_of(const float* c) {
    Camera cam;
    static_assert(sizeof(Vector3float) == 12, "layout");
    std::memcpy(reinterpret_cast<void*>(&cam), c, 12 * sizeof(float));
    return cam;
}

struct RadiancePayload {  // PathTracer.cu:11-18
    uint32_t seed;
    Vector3float radiance = 0;
    Vector3float rayweight = 1;
    Vector3float out_dir;
    bool next_ray_valid = false;
};

// PathTracer.cu:20-26
void emissive(Ray& ray, LocalGeometry& geom) {
    RadiancePayload* p = ray.payload<RadiancePayload>();
    p->radiance += p->rayweight * geom.material.albedo_e;
}

// PathTracer.cu:28-74
void direct(Scene& scene, Ray& ray, LocalGeometry& geom, Vector3float& inc_dir, uint64_t& shadow_rays) {
    RadiancePayload* p = ray.payload<RadiancePayload>();
    Vector3float normal = geom.N;
    if (geom.material.type != MaterialType::GLASS && Math::dot(normal, inc_dir) <= 0.0f) {
        p->rayweight = 0;
        return;
    }
    uint32_t useEnv = scene.useEnvironmentMap ? 1 : 0;
    uint32_t light_sample = static_cast<uint32_t>(Math::rnd(p->seed) * (scene.light_count + useEnv));
    Light light;
    Vector3float lightDir, lightRadiance;
    float d;
    if (light_sample != scene.light_count) {
        light = *(scene.lights[light_sample]);
        lightRadiance = light.sample(p->seed, geom.P, lightDir, d);
    } else {
        Vector4float sample = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
        lightDir = Vector3float(sample);
        d = INFINITY;
        if (useEnv) {
            Vector2uint32_t pixel = Tracing::direction2UV(lightDir, scene.environment.width(), scene.environment.height());
            lightRadiance = scene.environment(pixel) / sample.w;
        } else {
            lightRadiance = 0;  // the reference reads an empty image here
        }
    }
    Ray shadow_ray = Ray(geom.P + 0.001f * lightDir, lightDir);
    ++shadow_rays;
    if (Tracing::traceVisibility(scene, d, shadow_ray)) {
        p->radiance += (scene.light_count + useEnv) * fmaxf(0.0f, Math::dot(normal, lightDir)) *
                       geom.material.brdf(geom.P, inc_dir, lightDir, normal) * lightRadiance * p->rayweight;
    }
}

// PathTracer.cu:76-95
void indirect(Ray& ray, LocalGeometry& geom, Vector3float& inc_dir) {
    RadiancePayload* p = ray.payload<RadiancePayload>();
    Vector4float direction_p = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
    Vector3float direction = Vector3float(direction_p);
    if (Math::norm(direction) < EPSILON) return;
    p->rayweight = p->rayweight * std::fabs(Math::dot(direction, geom.N)) *
                   geom.material.brdf(geom.P, inc_dir, direction, geom.N) / direction_p.w;
    p->out_dir = direction;
    p->next_ray_valid = true;
}

// PathTracer.cu:97-169 for one thread id.
Vector3float path(Scene& scene, const Camera& camera, uint32_t tid, uint32_t w, uint32_t h, uint32_t frameIndex,
                  uint32_t maxTraceDepth, bool useRR, uint64_t& ext, uint64_t& shd) {
    uint32_t seed = Math::tea<4>(tid, frameIndex);
    Ray ray = Tracing::launchRay(tid, w, h, camera, true, &seed);
    RadiancePayload payload;
    payload.seed = seed;
    ray.setPayload(&payload);
    uint32_t trace_depth = 0;
    do {
        payload.next_ray_valid = false;
        LocalGeometry geom = Tracing::traceRay(scene, ray);
        ++ext;
        if (geom.depth == INFINITY) {
            if (scene.useEnvironmentMap) {
                Vector2uint32_t pixel = Tracing::direction2UV(ray.direction(), scene.environment.width(), scene.environment.height());
                payload.radiance += payload.rayweight * scene.environment(pixel);
            }
            break;
        }
        Vector3float inc_dir = -1.0f * ray.direction();
        emissive(ray, geom);
        direct(scene, ray, geom, inc_dir, shd);
        if (useRR) {
            float alpha = Math::clamp(fmaxf(payload.rayweight.x, fmaxf(payload.rayweight.y, payload.rayweight.z)), 0.0f, 1.0f);
            if (Math::rnd(payload.seed) > alpha || Math::safeFloatEqual(alpha, 0)) {
                payload.next_ray_valid = false;
                payload.rayweight = 0;
                break;
            }
            payload.rayweight = payload.rayweight / alpha;
        }
        indirect(ray, geom, inc_dir);
        ray.traceNew(geom.P + 0.01f * payload.out_dir, payload.out_dir);
        if (!payload.next_ray_valid) break;
        ++trace_depth;
    } while (trace_depth < maxTraceDepth);
    return payload.radiance;
}

// ------------------------------------------------------------ VOLUME ---
// VolumeRenderer.cu:11-310.  The reference stores the current medium as a
// pointer into the loop-local LocalGeometry; here the medium is held by
// value: the volume of the object the path is inside (every hit while
// inside is on that object), the scene volume outside.
struct VolPayload {  // VolumeRenderer.cu:11-22
    uint32_t seed;
    Vector3float radiance = 0;
    Vector3float rayweight = 1;
    Vector3float ray_start;
    Vector3float out_dir;
    bool next_ray_valid;
    Volume volume;
    bool inside_object = false;
    uint32_t object_index = 0;
};

void direct_vol(Scene& scene, VolPayload* p, LocalGeometry& geom, Vector3float& inc_dir) {  // :24-70
    Vector3float normal = geom.N;
    if (geom.material.type != MaterialType::GLASS && Math::dot(normal, inc_dir) <= 0.0f) {
        p->rayweight = 0;
        return;
    }
    uint32_t useEnv = scene.useEnvironmentMap ? 1 : 0;
    uint32_t light_sample = static_cast<uint32_t>(Math::rnd(p->seed) * (scene.light_count + useEnv));
    Light light;
    Vector3float lightDir, lightRadiance;
    float d;
    if (light_sample != scene.light_count) {
        light = *(scene.lights[light_sample]);
        lightRadiance = light.sample(p->seed, geom.P, lightDir, d);
    } else {
        Vector4float sample = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
        lightDir = Vector3float(sample);
        d = INFINITY;
        if (useEnv) {
            Vector2uint32_t pixel = Tracing::direction2UV(lightDir, scene.environment.width(), scene.environment.height());
            lightRadiance = scene.environment(pixel) / sample.w;
        } else {
            lightRadiance = 0;
        }
    }
    Ray shadow_ray = Ray(geom.P + 0.001f * lightDir, lightDir);
    if (Tracing::traceVisibility(scene, d, shadow_ray)) {
        p->radiance += (scene.light_count + useEnv) * fmaxf(0.0f, Math::dot(normal, lightDir)) *
                       Math::exp(-1.0f * (p->volume.sigma_s + p->volume.sigma_a) * fminf(d, 100000000.0f)) *
                       geom.material.brdf(geom.P, inc_dir, lightDir, normal) * lightRadiance * p->rayweight;
    }
}

void indirect_vol(VolPayload* p, LocalGeometry& geom, Vector3float& inc_dir) {  // :72-86
    Vector4float direction_p = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
    Vector3float direction = Vector3float(direction_p);
    if (Math::norm(direction) == 0) return;
    p->rayweight = p->rayweight * std::fabs(Math::dot(direction, geom.N)) *
                   geom.material.brdf(geom.P, inc_dir, direction, geom.N) / direction_p.w;
    p->out_dir = direction;
    p->ray_start = geom.P;
    p->next_ray_valid = true;
}

bool medium_vol(Scene& scene, Ray& ray, VolPayload* p, LocalGeometry& geom, Vector3float& inc_dir) {  // :88-212
    float g = p->volume.g;
    Vector3float sigma_a = p->volume.sigma_a;
    Vector3float sigma_s = p->volume.sigma_s;
    Vector3float sigma_t = sigma_a + sigma_s;
    uint32_t channel = static_cast<uint32_t>(Math::rnd(p->seed) * 3);
    if (Math::safeFloatEqual(sigma_t[channel], 0.0f)) return false;
    float t = -logf(1.0f - Math::rnd(p->seed)) / sigma_t[channel];
    if (t < geom.depth) {
        Vector3float event_position = ray.origin() + t * ray.direction();
        float scattering_prob = sigma_s[channel] / sigma_t[channel];
        if (Math::rnd(p->seed) < scattering_prob) {
            float pdf = 0.0f;
            for (uint32_t i = 0; i < 3; ++i) pdf += sigma_t[i] * expf(-1.0f * sigma_t[i] * t);
            pdf /= 3.0f;
            p->rayweight = p->rayweight * sigma_s / scattering_prob * Math::exp(-1.0f * sigma_t * t) / pdf;
        } else {
            p->rayweight = 0;
            p->next_ray_valid = false;
            return true;
        }
        uint32_t useEnv = scene.useEnvironmentMap ? 1 : 0;
        uint32_t light_sample = static_cast<uint32_t>(Math::rnd(p->seed) * (scene.light_count + useEnv));
        Light light;
        Vector3float lightDir, lightRadiance;
        float d;
        if (light_sample != scene.light_count) {
            light = *(scene.lights[light_sample]);
            lightRadiance = light.sample(p->seed, event_position, lightDir, d);
        } else {
            Vector4float sample = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
            lightDir = Vector3float(sample);
            d = INFINITY;
            if (useEnv) {
                Vector2uint32_t pixel = Tracing::direction2UV(lightDir, scene.environment.width(), scene.environment.height());
                lightRadiance = scene.environment(pixel) / sample.w;
            } else {
                lightRadiance = 0;
            }
        }
        Ray shadow_ray;
        Vector3float attenuation = 1.0f;
        if (p->inside_object) {
            shadow_ray = Ray(event_position, lightDir);
            LocalGeometry ge = Tracing::traceRay(scene, shadow_ray, p->object_index);
            if (ge.depth == INFINITY) {
                ge.depth = 0;
                ge.P = event_position;
            }
            attenuation = Math::exp(-1.0f * sigma_t * ge.depth) *
                          Material::henyeyGreensteinPhaseFunction(g, -Math::dot(inc_dir, lightDir));
            shadow_ray.traceNew(ge.P + 0.001f * lightDir, lightDir);
            d -= ge.depth;
        } else {
            shadow_ray = Ray(event_position + 0.001f * lightDir, lightDir);
        }
        Vector3float scene_sigma_t = scene.volume.sigma_a + scene.volume.sigma_s;
        if (Tracing::traceVisibility(scene, d, shadow_ray)) {
            p->radiance += (float)(scene.light_count + useEnv) * Math::exp(-1.0f * scene_sigma_t * fminf(d, 100000000.0f)) *
                           attenuation * lightRadiance * p->rayweight;
        }
        Vector4float sample_hg = sampleHenyeyGreensteinPhaseFunction(g, -1.0f * inc_dir, p->seed);
        p->out_dir = Vector3float(sample_hg);
        p->ray_start = event_position;
        p->next_ray_valid = true;
        return true;
    }
    float pdf = 0.0f;
    for (uint32_t i = 0; i < 3; ++i) pdf += expf(-sigma_t[i] * geom.depth);
    pdf /= 3.0f;
    p->rayweight = p->rayweight * Math::exp(-1.0f * sigma_t * geom.depth) / pdf;
    p->ray_start = geom.P;
    return false;
}

Vector3float volume_path(Scene& scene, const Camera& camera, uint32_t tid, uint32_t w, uint32_t h, uint32_t frameIndex,
                         uint32_t maxTraceDepth, bool useRR) {  // :214-310
    uint32_t seed = Math::tea<4>(tid, frameIndex);
    Ray ray = Tracing::launchRay(tid, w, h, camera, true, &seed);
    VolPayload payload;
    payload.seed = seed;
    payload.volume = scene.volume;
    uint32_t trace_depth = 0;
    do {
        payload.next_ray_valid = false;
        LocalGeometry geom;
        if (!payload.inside_object) geom = Tracing::traceRay(scene, ray);
        else geom = Tracing::traceRay(scene, ray, payload.object_index);
        Vector3float inc_dir = -1.0f * ray.direction();
        if (geom.depth == INFINITY) {
            if (scene.useEnvironmentMap) {
                Vector2uint32_t pixel = Tracing::direction2UV(ray.direction(), scene.environment.width(), scene.environment.height());
                payload.radiance += payload.rayweight * scene.environment(pixel);
            }
            break;
        }
        if (!medium_vol(scene, ray, &payload, geom, inc_dir)) {
            if (geom.material.type == MaterialType::VOLUME) {
                payload.out_dir = geom.material.sampleDirection(payload.seed, inc_dir, geom.N);
                payload.ray_start = geom.P;
                bool reflect = Math::dot(inc_dir, geom.N) * Math::dot(payload.out_dir, geom.N) > 0;
                payload.inside_object = reflect ? payload.inside_object : !payload.inside_object;
                payload.object_index = geom.scene_index;
                payload.next_ray_valid = true;
                payload.volume = payload.inside_object ? geom.material.volume : scene.volume;
            } else {
                direct_vol(scene, &payload, geom, inc_dir);
                indirect_vol(&payload, geom, inc_dir);
            }
            if (useRR) {
                float alpha = Math::clamp(fmaxf(payload.rayweight.x, fmaxf(payload.rayweight.y, payload.rayweight.z)), 0.0f, 1.0f);
                if (Math::rnd(payload.seed) > alpha || Math::safeFloatEqual(alpha, 0)) {
                    payload.next_ray_valid = false;
                    payload.rayweight = 0;
                    break;
                }
                payload.rayweight = payload.rayweight / alpha;
            }
        }
        ray.traceNew(payload.ray_start + 0.001f * payload.out_dir, payload.out_dir);
        if (!payload.next_ray_valid) break;
        ++trace_depth;
    } while (trace_depth < maxTraceDepth);
    return payload.radiance;
}

// ---------------------------------------------------- GRADIENTDOMAIN ---
// GradientDomain.cu:11-246; never-written base vertices count as invalid.
struct PathData {  // :15-23
    Vector3float position;
    Vector3float normal;
    bool diffuse;
    float pdf;
    bool valid = false;
};
struct GdPayload {  // :25-35
    uint32_t seed;
    Vector3float radiance = 0;
    Vector3float rayweight = 1;
    Vector3float out_dir;
    bool next_ray_valid;
    uint32_t trace_depth = 0;
    PathData path[64];
    PathData* base_path = nullptr;
    bool shift = false;
};

void collect(Ray& ray, Scene& scene, GdPayload* p, uint32_t maxTraceDepth) {  // :110-158
    uint32_t trace_depth = 0;
    do {
        p->next_ray_valid = false;
        if (p->shift && !p->base_path[p->trace_depth].valid) return;
        LocalGeometry geom = Tracing::traceRay(scene, ray);
        if (geom.depth == INFINITY) {
            p->path[p->trace_depth].valid = false;
            if (scene.useEnvironmentMap) {
                Vector2uint32_t pixel = Tracing::direction2UV(ray.direction(), scene.environment.width(), scene.environment.height());
                p->radiance += p->rayweight * scene.environment(pixel);
            }
            break;
        }
        p->path[p->trace_depth].position = geom.P;
        p->path[p->trace_depth].normal = geom.N;
        p->path[p->trace_depth].valid = true;
        p->path[p->trace_depth].diffuse = geom.material.shininess > 0.1f;
        Vector3float inc_dir = -1.0f * ray.direction();
        // emissiveIllumintationGDPT (:37-43)
        p->radiance += p->rayweight * geom.material.albedo_e;
        // directIlluminationGDPT (:45-91): same as the path tracer's
        {
            RadiancePayload rp;
            rp.seed = p->seed;
            rp.radiance = p->radiance;
            rp.rayweight = p->rayweight;
            Ray tmp = ray;
            tmp.setPayload(&rp);
            uint64_t shd = 0;
            direct(scene, tmp, geom, inc_dir, shd);
            p->seed = rp.seed;
            p->radiance = rp.radiance;
            p->rayweight = rp.rayweight;
        }
        // indirectIlluminationGDPT (:93-108)
        Vector4float direction_p = geom.material.sampleDirection(p->seed, inc_dir, geom.N);
        Vector3float direction = Vector3float(direction_p);
        if (!(Math::norm(direction) == 0)) {
            p->rayweight = p->rayweight * std::fabs(Math::dot(direction, geom.N)) *
                           geom.material.brdf(geom.P, inc_dir, direction, geom.N) / direction_p.w;
            p->out_dir = direction;
            p->next_ray_valid = true;
            p->path[p->trace_depth].pdf = direction_p.w;
        }
        ray.traceNew(geom.P + 0.01f * p->out_dir, p->out_dir);
        if (!p->next_ray_valid) break;
        ++trace_depth;
        ++p->trace_depth;
    } while (trace_depth < maxTraceDepth);
}

}  // namespace

extern "C" {

void* ref_scene_new() { return new RefScene(); }

// raytracing_kernel (RayTracer.cu:11-54) for all w*h pixels
void ref_raytrace(void* s, const float* cam, uint32_t w, uint32_t h, float* img) {
    RefScene* r = static_cast<RefScene*>(s);
    Scene& scene = r->scene;
    Camera camera = camera_of(cam);
    for (uint32_t tid = 0; tid < w * h; ++tid) {
        Ray ray = Tracing::launchRay(tid, w, h, camera);
        LocalGeometry geom = Tracing::traceRay(scene, ray);
        Vector3float inc_dir = Math::normalize(camera.position() - geom.P);
        Vector3float radiance = 0;
        for (uint32_t i = 0; i < scene.light_count; ++i) {
            Vector3float lightDir = Math::normalize(scene.lights[i]->position - geom.P);
            Vector3float brdf = geom.material.brdf(geom.P, inc_dir, lightDir, geom.N);
            float d = Math::norm(geom.P - scene.lights[i]->position);
            Vector3float lightRadiance = scene.lights[i]->intensity / (d * d);
            float cosTerm = std::max(0.0f, Math::dot(geom.N, lightDir));
            if (geom.depth != INFINITY) {
                Ray shadow_ray(geom.P - EPSILON * ray.direction(), lightDir);
                if (Tracing::traceVisibility(scene, d, shadow_ray)) radiance += brdf * lightRadiance * cosTerm;
            }
        }
        img[3 * tid] = radiance.x;
        img[3 * tid + 1] = radiance.y;
        img[3 * tid + 2] = radiance.z;
    }
}

// volume_kernel running mean (VolumeRenderer.cu:214-310)
void ref_volumetrace(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                     uint32_t maxDepth, int rr, float* img) {
    RefScene* r = static_cast<RefScene*>(s);
    Camera camera = camera_of(cam);
    for (uint32_t i = 0; i < w * h; ++i) {
        Vector3float acc(img[3 * i], img[3 * i + 1], img[3 * i + 2]);
        for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
            Vector3float rad = volume_path(r->scene, camera, i, w, h, f, maxDepth, rr != 0);
            if (f > 0) {
                const float a = 1.0f / (static_cast<float>(f) + 1.0f);
                rad = (1.0f - a) * acc + a * rad;
            }
            acc = rad;
        }
        img[3 * i] = acc.x;
        img[3 * i + 1] = acc.y;
        img[3 * i + 2] = acc.z;
    }
}

// gdpt_kernel frames (GradientDomain.cu:160-246): running means of base and
// the four one-sided gradients.
void ref_gdpt_frames(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                     uint32_t maxDepth, float* base, float* gxf, float* gxb, float* gyf, float* gyb) {
    RefScene* r = static_cast<RefScene*>(s);
    Camera camera = camera_of(cam);
    float* imgs[5] = {base, gxf, gxb, gyf, gyb};
    for (uint32_t tid = 0; tid < w * h; ++tid) {
        const Vector2int32_t pixel = ThreadHelper::index2pixel(tid, w, h);
        if (pixel.x == 0 || pixel.x == (int)w - 1 || pixel.y == 0 || pixel.y == (int)h - 1) continue;
        for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
            uint32_t seed = Math::tea<4>(tid, f);
            GdPayload pl[5];
            Ray rays[5];
            const Vector2int32_t off[5] = {Vector2int32_t(0, 0), Vector2int32_t(-1, 0), Vector2int32_t(1, 0),
                                           Vector2int32_t(0, 1), Vector2int32_t(0, -1)};
            for (int k = 0; k < 5; ++k) {
                Vector2uint32_t px = pixel + off[k];
                rays[k] = Tracing::launchRay(px, w, h, camera, true, &seed);
                pl[k].seed = seed;
                if (k > 0) {
                    pl[k].base_path = pl[0].path;
                    pl[k].shift = true;
                }
            }
            for (int k = 0; k < 5; ++k) collect(rays[k], r->scene, &pl[k], maxDepth);
            Vector3float radiance = pl[0].radiance;
            Vector3float out[5] = {radiance, 0.5f * (radiance - pl[1].radiance), 0.5f * (pl[2].radiance - radiance),
                                   0.5f * (radiance - pl[4].radiance), 0.5f * (pl[3].radiance - radiance)};
            for (int k = 0; k < 5; ++k) {
                float* q = imgs[k] + 3 * (size_t)tid;
                Vector3float v = out[k];
                if (f > 0) {
                    const float a = 1.0f / (static_cast<float>(f) + 1.0f);
                    v = (1.0f - a) * Vector3float(q[0], q[1], q[2]) + a * v;
                }
                q[0] = v.x;
                q[1] = v.y;
                q[2] = v.z;
            }
        }
    }
}

void ref_scene_free(void* s) { delete static_cast<RefScene*>(s); }  // geometry is leaked on purpose (tests only)

// Same flat layouts as oracle/oracle_capi.cpp.
void ref_scene_add_object(void* s, int type, const float* geo, float radius, const float* mat, const float* tris,
                          int ntris, const float* box) {
    RefScene* r = static_cast<RefScene*>(s);
    Geometry* g = nullptr;
    switch (type) {
        case 0: g = new Sphere(v3(geo), radius); break;                          // SceneLoader.cpp:199-210
        case 1: g = new Plane(v3(geo), v3(geo + 3)); break;                      // :186-198
        case 2: g = new Quad(v3(geo), v3(geo + 3), v3(geo + 6), v3(geo + 9)); break;  // :211-228
        case 3: g = new Triangle(v3(tris), v3(tris + 3), v3(tris + 6)); break;   // :229-244
        case 4: {                                                               // ObjLoader.cpp:67-85
            Triangle* buf = new Triangle[ntris];
            for (int i = 0; i < ntris; ++i) {
                const float* t = tris + 9 * (size_t)i;
                buf[i] = Triangle(v3(t), v3(t + 3), v3(t + 6));
            }
            g = new Mesh(buf, (uint32_t)ntris, v3(box), v3(box + 3));
            break;
        }
    }
    g->material = material_of(mat);
    g->setID((uint32_t)r->geometry.size());
    r->geometry.push_back(g);
}

void ref_scene_add_light(void* s, const float* l) {
    RefScene* r = static_cast<RefScene*>(s);
    Light* li = new Light();
    li->type = (int)l[0] == 0 ? POINT : AREA;
    li->position = v3(l + 1);
    li->intensity = v3(l + 4);
    li->radiance = v3(l + 7);
    li->halfExtend1 = v3(l + 10);
    li->halfExtend2 = v3(l + 13);
    r->lights.push_back(li);
}

void ref_scene_set_env(void* s, const float* rgb, uint32_t w, uint32_t h) {
    RefScene* r = static_cast<RefScene*>(s);
    Image<Vector3float> img = Image<Vector3float>::createHostObject(w, h);
    for (size_t i = 0; i < (size_t)w * h; ++i) img[(unsigned)i] = v3(rgb + 3 * i);
    r->scene.environment = img;
    r->scene.useEnvironmentMap = true;
}

void ref_scene_set_volume(void* s, const float* sigma_s, const float* sigma_a, float g) {  // SceneLoader.cpp:330-344
    RefScene* r = static_cast<RefScene*>(s);
    Volume vol;
    vol.sigma_s = v3(sigma_s);
    vol.sigma_a = v3(sigma_a);
    vol.g = g;
    r->scene.volume = vol;
}

void ref_scene_finalize(void* s) {
    RefScene* r = static_cast<RefScene*>(s);
    // SceneLoader.cpp:416-420 with "device" pointers that are host pointers
    BoundingVolumeHierarchy bvh(r->geometry, r->geometry);
    r->bvh = new BoundingVolumeHierarchy(bvh);
    r->scene.bvh = r->bvh;
    r->scene.geometry = r->geometry.data();
    r->scene.scene_size = (uint32_t)r->geometry.size();
    r->scene.lights = r->lights.data();
    r->scene.light_count = (uint32_t)r->lights.size();
}

// Tracing::traceRay (TracingDetail.h:47-66) for n rays.
void ref_trace(void* s, int n, const float* o, const float* d, float* t, int* obj, float* P, float* N) {
    RefScene* r = static_cast<RefScene*>(s);
    for (int i = 0; i < n; ++i) {
        Ray ray(v3(o + 3 * i), v3(d + 3 * i));
        LocalGeometry g = Tracing::traceRay(r->scene, ray);
        t[i] = g.depth;
        obj[i] = g.depth == INFINITY ? -1 : g.scene_index;
        if (P) { P[3 * i] = g.P.x; P[3 * i + 1] = g.P.y; P[3 * i + 2] = g.P.z; }
        if (N) { N[3 * i] = g.N.x; N[3 * i + 1] = g.N.y; N[3 * i + 2] = g.N.z; }
    }
}

// Tracing::traceVisibility (TracingDetail.h:118-183)
void ref_visible(void* s, int n, const float* o, const float* d, const float* dist, int* vis) {
    RefScene* r = static_cast<RefScene*>(s);
    for (int i = 0; i < n; ++i) {
        Ray ray(v3(o + 3 * i), v3(d + 3 * i));
        vis[i] = Tracing::traceVisibility(r->scene, dist[i], ray) ? 1 : 0;
    }
}

// Running-mean NEE path tracing of frames [frame0, frame0 + nframes) for the
// listed pixels (or all w*h when pixels == NULL), PathTracer.cu:162-168.
void ref_pathtrace(void* s, const float* cam, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                   uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img, int nthreads,
                   uint64_t* ray_counts) {
    RefScene* r = static_cast<RefScene*>(s);
    Camera camera = camera_of(cam);
    const int64_t n = pixels ? npix : (int64_t)w * h;
    std::atomic<uint64_t> ext_total{0}, shd_total{0};
    std::atomic<int64_t> next{0};
    // std::thread workers (no OpenMP: the library is loaded next to PyTorch's runtime)
    auto worker = [&]() {
        uint64_t ext = 0, shd = 0;
        for (;;) {
            int64_t b = next.fetch_add(8);
            if (b >= n) break;
            for (int64_t i = b; i < std::min(n, b + 8); ++i) {
                uint32_t tid = pixels ? pixels[i] : (uint32_t)i;
                Vector3float acc(img[3 * i], img[3 * i + 1], img[3 * i + 2]);
                for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
                    Vector3float rad = path(r->scene, camera, tid, w, h, f, maxDepth, rr != 0, ext, shd);
                    if (f > 0) {  // PathTracer.cu:162-168
                        const float a = 1.0f / (static_cast<float>(f) + 1.0f);
                        rad = (1.0f - a) * acc + a * rad;
                    }
                    acc = rad;
                }
                img[3 * i] = acc.x;
                img[3 * i + 1] = acc.y;
                img[3 * i + 2] = acc.z;
            }
        }
        ext_total += ext;
        shd_total += shd;
    };
    int nt = std::max(1, nthreads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (ray_counts) { ray_counts[0] = ext_total.load(); ray_counts[1] = shd_total.load(); }
}

// Math::tea<4> / Math::rnd (FunctionsDetail.h:70-98)
uint32_t ref_tea4(uint32_t a, uint32_t b) { return Math::tea<4>(a, b); }
void ref_rnd_stream(uint32_t seed, int n, float* out, uint32_t* states) {
    for (int i = 0; i < n; ++i) {
        out[i] = Math::rnd(seed);
        if (states) states[i] = seed;
    }
}

// Material::sampleDirection / brdf (MaterialDetail.h:35-111)
void ref_sample_direction(const float* m, uint32_t seed, const float* inc, const float* n, float* out4, uint32_t* seed_out) {
    Material mat = material_of(m);
    Vector4float r = mat.sampleDirection(seed, v3(inc), v3(n));
    out4[0] = r.x; out4[1] = r.y; out4[2] = r.z; out4[3] = r.w;
    if (seed_out) *seed_out = seed;
}
void ref_brdf(const float* m, const float* inc, const float* out, const float* n, float* res3) {
    Material mat = material_of(m);
    Vector3float r = mat.brdf(Vector3float(0), v3(inc), v3(out), v3(n));
    res3[0] = r.x; res3[1] = r.y; res3[2] = r.z;
}
// Light::sample (LightDetail.h:8-52)
void ref_light_sample(const float* l, uint32_t seed, const float* P, float* rad3, float* dir3, float* dist, uint32_t* seed_out) {
    Light li;
    li.type = (int)l[0] == 0 ? POINT : AREA;
    li.position = v3(l + 1);
    li.intensity = v3(l + 4);
    li.radiance = v3(l + 7);
    li.halfExtend1 = v3(l + 10);
    li.halfExtend2 = v3(l + 13);
    Vector3float dir;
    float d;
    Vector3float r = li.sample(seed, v3(P), dir, d);
    rad3[0] = r.x; rad3[1] = r.y; rad3[2] = r.z;
    dir3[0] = dir.x; dir3[1] = dir.y; dir3[2] = dir.z;
    *dist = d;
    if (seed_out) *seed_out = seed;
}

}  // extern "C"
