// Device build of the REFERENCE's own CUDA path (test and reference-arm infrastructure).
//
// Compiled by oracle/build_oracle.py with nvcc for sm_100a and -use_fast_math
// (the reference's only CUDA flag, CMakeLists.txt:61) against the reference
// sources where they lie, into oracle/_ref/libref_cuda.so.  This driver only
// assembles a cupbr::Scene the way SceneLoader::loadFromFile does
// (SceneLoader.cpp:370-453: per-object device copies, mesh triangle arrays,
// the object BVH constructor, device pointer tables) from flat arrays, and
// then calls the reference's own entry points:
//   PBRendering::pathtracing      (PathTracer.cu:260-276, kernel :97-169)
//   PostProcessor::bloom          (PostProcessor.cpp:125-142)
//   ToneMapper::toneMap           (ToneMapper.cu:132-181)
// It is used to time the reference's CUDA path on the same GPU and to compare
// its (fast-math) images with the cupbr-b200 kernels.
#include <cstdint>
#include <cstring>
#include <vector>

#include <DataStructure/BoundingVolumeHierarchy.h>
#include <DataStructure/Camera.h>
#include <DataStructure/Image.h>
#include <DataStructure/Light.h>
#include <Geometry/Mesh.h>
#include <Geometry/Plane.h>
#include <Geometry/Quad.h>
#include <Geometry/Sphere.h>
#include <Geometry/Triangle.h>
#include <PostProcessing/PostProcessor.h>
#include <Renderer/GradientDomain.h>
#include <Renderer/PathTracer.h>
#include <Renderer/RayTracer.h>
#include <Renderer/ToneMapper.h>
#include <Renderer/VolumeRenderer.h>
#include <Scene/Scene.h>

using namespace cupbr;

namespace {

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

struct RefCudaScene {
    Scene scene;
    std::vector<Geometry*> host_geo;
    std::vector<Light*> host_lights;
    Image<Vector3float> env;
    bool has_env = false;
    cudaError_t err = cudaSuccess;
};

template <typename T>
Geometry* to_device(T* host_obj) {  // SceneLoader.cpp:372-414
    T* dev = Memory::createDeviceObject<T>();
    Memory::copyHost2DeviceObject<T>(host_obj, dev);
    return dev;
}

}  // namespace

extern "C" {

void* refcu_scene_new() { return new RefCudaScene(); }

void refcu_scene_add_object(void* s, int type, const float* geo, float radius, const float* mat, const float* tris,
                            int ntris, const float* box) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Geometry* g = nullptr;
    switch (type) {
        case 0: g = new Sphere(v3(geo), radius); break;
        case 1: g = new Plane(v3(geo), v3(geo + 3)); break;
        case 2: g = new Quad(v3(geo), v3(geo + 3), v3(geo + 6), v3(geo + 9)); break;
        case 3: g = new Triangle(v3(tris), v3(tris + 3), v3(tris + 6)); break;
        case 4: {  // ObjLoader.cpp:67-85: triangle array on the device, Mesh on the host
            std::vector<Triangle> host(ntris);
            for (int i = 0; i < ntris; ++i) {
                const float* t = tris + 9 * (size_t)i;
                host[i] = Triangle(v3(t), v3(t + 3), v3(t + 6));
            }
            Triangle* dev_tris = Memory::createDeviceArray<Triangle>((uint32_t)ntris);
            Memory::copyHost2DeviceArray<Triangle>((uint32_t)ntris, host.data(), dev_tris);
            g = new Mesh(dev_tris, (uint32_t)ntris, v3(box), v3(box + 3));
            break;
        }
    }
    g->material = material_of(mat);
    g->setID((uint32_t)r->host_geo.size());
    r->host_geo.push_back(g);
}

void refcu_scene_add_light(void* s, const float* l) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Light* li = new Light();
    li->type = (int)l[0] == 0 ? POINT : AREA;
    li->position = v3(l + 1);
    li->intensity = v3(l + 4);
    li->radiance = v3(l + 7);
    li->halfExtend1 = v3(l + 10);
    li->halfExtend2 = v3(l + 13);
    r->host_lights.push_back(li);
}

void refcu_scene_set_env(void* s, const float* rgb, uint32_t w, uint32_t h) {  // SceneLoader.cpp:346-368
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Image<Vector3float> buffer = Image<Vector3float>::createHostObject(w, h);
    for (size_t i = 0; i < (size_t)w * h; ++i) buffer[(unsigned)i] = v3(rgb + 3 * i);
    Image<Vector3float> dbuffer = Image<Vector3float>::createDeviceObject(w, h);
    buffer.copyHost2DeviceObject(dbuffer);
    r->scene.useEnvironmentMap = true;
    r->scene.environment = dbuffer;
    Image<Vector3float>::destroyHostObject(buffer);
}

int refcu_scene_finalize(void* s) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Scene& sc = r->scene;
    sc.scene_size = (uint32_t)r->host_geo.size();
    sc.light_count = (uint32_t)r->host_lights.size();
    sc.geometry = Memory::createDeviceArray<Geometry*>(sc.scene_size);
    sc.lights = Memory::createDeviceArray<Light*>(sc.light_count);
    std::vector<Geometry*> dev;
    for (Geometry* g : r->host_geo) {
        switch (g->type) {
            case GeometryType::SPHERE: dev.push_back(to_device(static_cast<Sphere*>(g))); break;
            case GeometryType::PLANE: dev.push_back(to_device(static_cast<Plane*>(g))); break;
            case GeometryType::QUAD: dev.push_back(to_device(static_cast<Quad*>(g))); break;
            case GeometryType::TRIANGLE: dev.push_back(to_device(static_cast<Triangle*>(g))); break;
            default: dev.push_back(to_device(static_cast<Mesh*>(g))); break;
        }
    }
    BoundingVolumeHierarchy bvh(r->host_geo, dev);  // SceneLoader.cpp:416-418
    sc.bvh = Memory::createDeviceObject<BoundingVolumeHierarchy>();
    Memory::copyHost2DeviceObject<BoundingVolumeHierarchy>(&bvh, sc.bvh);
    Memory::copyHost2DeviceArray(dev.size(), dev.data(), sc.geometry);
    std::vector<Light*> dl;
    for (Light* l : r->host_lights) {
        Light* d = Memory::createDeviceObject<Light>();
        Memory::copyHost2DeviceObject<Light>(l, d);
        dl.push_back(d);
    }
    Memory::copyHost2DeviceArray(dl.size(), dl.data(), sc.lights);
    return (int)cudaDeviceSynchronize();
}

// PBRendering::pathtracing for frames [frame0, frame0 + nframes) into a
// running-mean image; img (w*h*3 host floats) is the starting image and
// receives the result; *ms = summed CUDA-event time of the render calls.
int refcu_pathtrace(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                    uint32_t max_depth, int rr, float* img, float* ms) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Camera camera;
    std::memcpy(reinterpret_cast<void*>(&camera), cam, 12 * sizeof(float));
    Image<Vector3float> out = Image<Vector3float>::createDeviceObject(w, h);
    cudaMemcpy(out.data(), img, sizeof(float) * 3 * (size_t)w * h, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (uint32_t f = frame0; f < frame0 + nframes; ++f)
        PBRendering::pathtracing(r->scene, camera, f, max_depth, rr != 0, &out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaMemcpy(img, out.data(), sizeof(float) * 3 * (size_t)w * h, cudaMemcpyDeviceToHost);
    Image<Vector3float>::destroyDeviceObject(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaGetLastError();
}

void refcu_scene_set_volume(void* s, const float* sigma_s, const float* sigma_a, float g) {  // SceneLoader.cpp:330-344
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Volume vol;
    vol.sigma_s = v3(sigma_s);
    vol.sigma_a = v3(sigma_a);
    vol.g = g;
    r->scene.volume = vol;
}

// PBRendering::volumetracing (VolumeRenderer.cu:313-329) frames into img
int refcu_volumetrace(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                      uint32_t max_depth, int rr, float* img, float* ms) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Camera camera;
    std::memcpy(reinterpret_cast<void*>(&camera), cam, 12 * sizeof(float));
    Image<Vector3float> out = Image<Vector3float>::createDeviceObject(w, h);
    cudaMemcpy(out.data(), img, sizeof(float) * 3 * (size_t)w * h, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (uint32_t f = frame0; f < frame0 + nframes; ++f)
        PBRendering::volumetracing(r->scene, camera, f, max_depth, rr != 0, &out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaMemcpy(img, out.data(), sizeof(float) * 3 * (size_t)w * h, cudaMemcpyDeviceToHost);
    Image<Vector3float>::destroyDeviceObject(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaGetLastError();
}

// PBRendering::gradientdomain (GradientDomain.cu:353-402) frames; buffers
// cleared first as PBRenderer::setMethod does (PBRenderer.cu:118-135).
// out9 receives (host, w*h*3 each): output, gradient_x, gradient_y, base,
// gx_forward, gx_backward, gy_forward, gy_backward, temp.
int refcu_gradientdomain(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                         uint32_t max_depth, float* out9, float* ms) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Camera camera;
    std::memcpy(reinterpret_cast<void*>(&camera), cam, 12 * sizeof(float));
    const size_t n = (size_t)w * h;
    Image<Vector3float> img[9];
    for (int k = 0; k < 9; ++k) {
        img[k] = Image<Vector3float>::createDeviceObject(w, h);
        cudaMemset(img[k].data(), 0, sizeof(float) * 3 * n);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (uint32_t f = frame0; f < frame0 + nframes; ++f)
        PBRendering::gradientdomain(r->scene, camera, f, max_depth, &img[3], &img[8], &img[1], &img[2], &img[4],
                                    &img[5], &img[6], &img[7], &img[0]);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    for (int k = 0; k < 9; ++k) {
        cudaMemcpy(out9 + 3 * n * k, img[k].data(), sizeof(float) * 3 * n, cudaMemcpyDeviceToHost);
        Image<Vector3float>::destroyDeviceObject(img[k]);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaGetLastError();
}

// PBRendering::raytracing (RayTracer.cu:57-64)
int refcu_raytrace(void* s, const float* cam, uint32_t w, uint32_t h, float* img) {
    RefCudaScene* r = static_cast<RefCudaScene*>(s);
    Camera camera;
    std::memcpy(reinterpret_cast<void*>(&camera), cam, 12 * sizeof(float));
    Image<Vector3float> out = Image<Vector3float>::createDeviceObject(w, h);
    PBRendering::raytracing(r->scene, camera, &out);
    cudaMemcpy(img, out.data(), sizeof(float) * 3 * (size_t)w * h, cudaMemcpyDeviceToHost);
    Image<Vector3float>::destroyDeviceObject(out);
    return (int)cudaGetLastError();
}

// PostProcessor::bloom on a host image (w*h*3 floats) -> out
int refcu_bloom(const float* hdr, uint32_t w, uint32_t h, const float* th, float* out) {
    Image<Vector3float> img = Image<Vector3float>::createDeviceObject(w, h);
    cudaMemcpy(img.data(), hdr, sizeof(float) * 3 * (size_t)w * h, cudaMemcpyHostToDevice);
    {
        PostProcessor pp;
        pp.registerImage(&img);
        pp.bloom(Vector4float(th[0], th[1], th[2], th[3]));
        cudaMemcpy(out, pp.getPostProcessBuffer()->data(), sizeof(float) * 3 * (size_t)w * h, cudaMemcpyDeviceToHost);
    }
    Image<Vector3float>::destroyDeviceObject(img);
    return (int)cudaGetLastError();
}

// ToneMapper::toneMap on a host image -> out (w*h*4 bytes)
int refcu_tonemap(const float* hdr, uint32_t w, uint32_t h, int type, float exposure, uint8_t* out) {
    Image<Vector3float> img = Image<Vector3float>::createDeviceObject(w, h);
    cudaMemcpy(img.data(), hdr, sizeof(float) * 3 * (size_t)w * h, cudaMemcpyHostToDevice);
    {
        ToneMapper tm(type == 0 ? ToneMappingType::REINHARD : ToneMappingType::GAMMA);
        tm.setExposure(exposure);
        tm.registerImage(&img);
        tm.toneMap();
        RenderBuffer rb = tm.getRenderBuffer();
        cudaMemcpy(out, rb.data(), 4 * (size_t)w * h, cudaMemcpyDeviceToHost);
    }
    Image<Vector3float>::destroyDeviceObject(img);
    return (int)cudaGetLastError();
}

// PostProcessor::bloom followed by ToneMapper::toneMap on the bloomed
// image, `iters` times on one uploaded image, timed with CUDA events:
// ms2[0] = ms per bloom, ms2[1] = ms per tone map.
int refcu_post_timed(const float* hdr, uint32_t w, uint32_t h, const float* th, int type, float exposure,
                     uint32_t iters, float* ms2) {
    Image<Vector3float> img = Image<Vector3float>::createDeviceObject(w, h);
    cudaMemcpy(img.data(), hdr, sizeof(float) * 3 * (size_t)w * h, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    {
        PostProcessor pp;
        pp.registerImage(&img);
        ToneMapper tm(type == 0 ? ToneMappingType::REINHARD : ToneMappingType::GAMMA);
        tm.setExposure(exposure);
        pp.bloom(Vector4float(th[0], th[1], th[2], th[3]));  // warm-up
        tm.registerImage(pp.getPostProcessBuffer());
        tm.toneMap();
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        for (uint32_t i = 0; i < iters; ++i) pp.bloom(Vector4float(th[0], th[1], th[2], th[3]));
        cudaEventRecord(e1);
        for (uint32_t i = 0; i < iters; ++i) tm.toneMap();
        cudaEventRecord(e2);
        cudaEventSynchronize(e2);
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&b, e1, e2);
        ms2[0] = a / (float)iters;
        ms2[1] = b / (float)iters;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    Image<Vector3float>::destroyDeviceObject(img);
    return (int)cudaGetLastError();
}

}  // extern "C"
