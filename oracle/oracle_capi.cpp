// C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY; see oracle.hpp).
//
// Built into oracle/liboracle.so by oracle/build_oracle.py and loaded with
// ctypes by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
// Layouts of the flat arrays:
//   material (20 floats): type, albedo_e[3], albedo_d[3], albedo_s[3],
//       shininess, roughness, eta, sigma_s[3], sigma_a[3], g     (+interface
//       passed separately as the 21st float: 1 = GLASS)
//   geometry (12 floats): p0[3], p1[3], p2[3], p3[3]
//       SPHERE: p0 = center            (radius separate)
//       PLANE : p0 = position, p1 = normal (normalized here, as the constructor does)
//       QUAD  : p0 = position, p1 = normal, p2 = extend1, p3 = extend2
//   triangles (9 floats each): v1, v2, v3 (already transformed)
//   light (16 floats): type, position[3], intensity[3], radiance[3], he1[3], he2[3]
//   camera (12 floats): position, x axis, y axis, z axis
#include "oracle.hpp"

#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <thread>

using namespace oracle;

namespace {

// std::thread parallel loop (no OpenMP: these libraries are loaded next to
// PyTorch, whose bundled OpenMP runtime shares the system runtime's soname).
int default_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n == 0 ? 1 : (int)n;
}
template <typename F>
void parallel_for(int64_t n, int64_t grain, int threads, F&& fn) {
    if (n <= 0) return;
    int nt = threads > 0 ? threads : default_threads();
    nt = (int)std::min<int64_t>(nt, (n + grain - 1) / grain);
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(grain);
            if (b >= n) break;
            fn(b, std::min(n, b + grain));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

struct AnyScene {
    int precision = 32;
    Scene<float> f;
    Scene<double> d;
};

template <typename R> V3<R> v3(const float* p) { return V3<R>(R(p[0]), R(p[1]), R(p[2])); }

template <typename R>
void add_object(Scene<R>& sc, int type, const float* geo, float radius, const float* mat, const float* tris, int ntris,
                const float* box) {
    Object<R> ob;
    ob.type = type;
    Material<R>& m = ob.mat;
    m.type = (int)mat[0];
    m.albedo_e = v3<R>(mat + 1);
    m.albedo_d = v3<R>(mat + 4);
    m.albedo_s = v3<R>(mat + 7);
    m.shininess = R(mat[10]);
    m.roughness = R(mat[11]);
    m.eta = R(mat[12]);
    m.sigma_s = v3<R>(mat + 13);
    m.sigma_a = v3<R>(mat + 16);
    m.g = R(mat[19]);
    m.interface_glass = mat[20] != 0.0f;
    ob.p0 = v3<R>(geo);
    ob.p1 = v3<R>(geo + 3);
    ob.p2 = v3<R>(geo + 6);
    ob.p3 = v3<R>(geo + 9);
    ob.radius = R(radius);
    // PlaneDetail.h:9-17, QuadDetail.h:9-19: the constructors normalize the normal
    if (type == PLANE || type == QUAD) ob.p1 = normalize(ob.p1);
    if (type == SPHERE) {  // SphereDetail.h:8-18
        ob.box_lo = ob.p0 - V3<R>(ob.radius);
        ob.box_hi = ob.p0 + V3<R>(ob.radius);
    }
    if (type == MESH || type == TRIANGLE) {
        ob.tris.reserve(ntris);
        for (int i = 0; i < ntris; ++i) {
            const float* t = tris + 9 * (size_t)i;
            ob.tris.push_back(make_tri(v3<R>(t), v3<R>(t + 3), v3<R>(t + 6)));
        }
    }
    if (type == MESH && box) {  // MeshDetail.h:11-19, box from ObjLoader.cpp:39-45
        ob.box_lo = v3<R>(box);
        ob.box_hi = v3<R>(box + 3);
    }
    sc.objects.push_back(std::move(ob));
}

template <typename R>
void add_light(Scene<R>& sc, const float* l) {
    Light<R> li;
    li.type = (int)l[0];
    li.position = v3<R>(l + 1);
    li.intensity = v3<R>(l + 4);
    li.radiance = v3<R>(l + 7);
    li.he1 = v3<R>(l + 10);
    li.he2 = v3<R>(l + 13);
    sc.lights.push_back(li);
}

template <typename R>
Camera<R> cam_of(const float* c) {
    Camera<R> cam;
    cam.pos = v3<R>(c);
    cam.xa = v3<R>(c + 3);
    cam.ya = v3<R>(c + 6);
    cam.za = v3<R>(c + 9);
    return cam;
}

template <typename R, typename OutT>
void pathtrace_impl(const Scene<R>& sc, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                    uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, OutT* img, int nthreads,
                    uint64_t* ray_counts, const ConstantCache<R>* cache = nullptr, int phys_mode = 0) {
    Camera<R> cam = cam_of<R>(camf);
    std::atomic<uint64_t> ext{0}, shd{0};
    parallel_for((int64_t)npix, 16, nthreads, [&](int64_t lo, int64_t hi) {
        RayStats st;
        for (int64_t i = lo; i < hi; ++i) {
            uint32_t tid = pixels ? pixels[i] : (uint32_t)i;
            V3<R> acc(R(img[3 * i + 0]), R(img[3 * i + 1]), R(img[3 * i + 2]));
            for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
                V3<R> rad = phys_mode ? trace_path_physical(sc, cam, tid, w, h, f, maxDepth, rr != 0, phys_mode, &st)
                                      : trace_path(sc, cam, tid, w, h, f, maxDepth, rr != 0, &st, cache);
                acc = running_mean(acc, rad, f);
            }
            img[3 * i + 0] = (OutT)acc.x;
            img[3 * i + 1] = (OutT)acc.y;
            img[3 * i + 2] = (OutT)acc.z;
        }
        ext += st.extension;
        shd += st.shadow;
    });
    if (ray_counts) { ray_counts[0] = ext.load(); ray_counts[1] = shd.load(); }
}

}  // namespace

extern "C" {

void* ora_scene_new(int precision) {
    AnyScene* s = new AnyScene();
    s->precision = precision == 64 ? 64 : 32;
    return s;
}
void ora_scene_free(void* s) { delete static_cast<AnyScene*>(s); }

void ora_scene_add_object(void* s, int type, const float* geo, float radius, const float* mat, const float* tris,
                          int ntris, const float* box) {
    AnyScene* a = static_cast<AnyScene*>(s);
    add_object(a->f, type, geo, radius, mat, tris, ntris, box);
    add_object(a->d, type, geo, radius, mat, tris, ntris, box);
}
void ora_scene_add_light(void* s, const float* l) {
    AnyScene* a = static_cast<AnyScene*>(s);
    add_light(a->f, l);
    add_light(a->d, l);
}
void ora_scene_set_env(void* s, const float* rgb, uint32_t w, uint32_t h) {
    AnyScene* a = static_cast<AnyScene*>(s);
    a->f.env_w = a->d.env_w = w;
    a->f.env_h = a->d.env_h = h;
    a->f.env.resize((size_t)w * h);
    a->d.env.resize((size_t)w * h);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        a->f.env[i] = v3<float>(rgb + 3 * i);
        a->d.env[i] = v3<double>(rgb + 3 * i);
    }
}
// Albedo texture (RGB, w * h, row v) and one object's planar projection.
void ora_scene_set_texture(void* s, const float* rgb, uint32_t w, uint32_t h) {
    AnyScene* a = static_cast<AnyScene*>(s);
    a->f.tex_w = a->d.tex_w = w;
    a->f.tex_h = a->d.tex_h = h;
    a->f.tex.resize((size_t)w * h);
    a->d.tex.resize((size_t)w * h);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        a->f.tex[i] = v3<float>(rgb + 3 * i);
        a->d.tex[i] = v3<double>(rgb + 3 * i);
    }
}
void ora_scene_set_object_texture(void* s, int obj, const float* origin, const float* u, const float* v) {
    AnyScene* a = static_cast<AnyScene*>(s);
    const float uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const float us[3] = {u[0] / uu, u[1] / uu, u[2] / uu}, vs[3] = {v[0] / vv, v[1] / vv, v[2] / vv};
    for (Object<float>* o : {&a->f.objects[obj]}) {
        o->textured = true;
        o->tex_o = v3<float>(origin);
        o->tex_u = v3<float>(us);
        o->tex_v = v3<float>(vs);
    }
    Object<double>& od = a->d.objects[obj];
    od.textured = true;
    od.tex_o = v3<double>(origin);
    od.tex_u = v3<double>(us);
    od.tex_v = v3<double>(vs);
}
void ora_scene_set_volume(void* s, const float* sigma_s, const float* sigma_a, float g) {
    AnyScene* a = static_cast<AnyScene*>(s);
    a->f.vol_sigma_s = v3<float>(sigma_s);
    a->f.vol_sigma_a = v3<float>(sigma_a);
    a->f.vol_g = g;
    a->d.vol_sigma_s = v3<double>(sigma_s);
    a->d.vol_sigma_a = v3<double>(sigma_a);
    a->d.vol_g = g;
}
void ora_scene_finalize(void* s) {
    AnyScene* a = static_cast<AnyScene*>(s);
    a->f.finalize();
    a->d.finalize();
}
int ora_scene_dfs_order(void* s, int* out, int cap) {
    AnyScene* a = static_cast<AnyScene*>(s);
    int n = (int)a->f.dfs_order.size();
    for (int i = 0; i < n && i < cap; ++i) out[i] = a->f.dfs_order[i];
    return n;
}

// Closest hit for n rays (directions are normalized as the Ray constructor
// does).  Outputs: depth (INF on miss), object id, triangle index, P, N.
void ora_trace(void* s, int n, const float* o, const float* d, float* t, int* obj, int* tri, float* P, float* N,
               int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    parallel_for(n, 64, nthreads, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            Ray<float> r(v3<float>(o + 3 * i), v3<float>(d + 3 * i));
            Hit<float> g = a->f.trace(r);
            t[i] = g.depth;
            obj[i] = g.obj;
            tri[i] = g.tri;
            if (P) { P[3 * i] = g.P.x; P[3 * i + 1] = g.P.y; P[3 * i + 2] = g.P.z; }
            if (N) { N[3 * i] = g.N.x; N[3 * i + 1] = g.N.y; N[3 * i + 2] = g.N.z; }
        }
    });
}

// Visibility (TracingDetail.h:118-183) for n rays with per-ray light distance.
void ora_visible(void* s, int n, const float* o, const float* d, const float* dist, int* vis, int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    parallel_for(n, 64, nthreads, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            Ray<float> r(v3<float>(o + 3 * i), v3<float>(d + 3 * i));
            vis[i] = a->f.visible(dist[i], r) ? 1 : 0;
        }
    });
}

// NEE path tracing (PathTracer.cu:97-169) of frames [frame0, frame0+nframes)
// into the running-mean image.  pixels == NULL renders all w*h pixels into
// img[w*h*3]; otherwise img holds npix rows for the listed pixel ids.
void ora_pathtrace_f32(void* s, const float* cam, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                       uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img, int nthreads,
                       uint64_t* ray_counts) {
    AnyScene* a = static_cast<AnyScene*>(s);
    pathtrace_impl(a->f, cam, w, h, pixels, pixels ? npix : w * h, frame0, nframes, maxDepth, rr, img, nthreads,
                   ray_counts);
}
void ora_pathtrace_f64(void* s, const float* cam, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                       uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, double* img, int nthreads,
                       uint64_t* ray_counts) {
    AnyScene* a = static_cast<AnyScene*>(s);
    pathtrace_impl(a->d, cam, w, h, pixels, pixels ? npix : w * h, frame0, nframes, maxDepth, rr, img, nthreads,
                   ray_counts);
}

// The physical estimators (trace_path_physical; mode PHYS_MIS, PHYS_NEE or
// PHYS_BSDF), running mean in float (precision 32) or double (64) into img.
void ora_pathtrace_phys(void* s, int precision, const float* cam, uint32_t w, uint32_t h, const uint32_t* pixels,
                        uint32_t npix, uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, int mode,
                        void* img, int nthreads, uint64_t* ray_counts) {
    AnyScene* a = static_cast<AnyScene*>(s);
    if (mode < PHYS_MIS || mode > PHYS_BSDF) mode = PHYS_MIS;
    if (precision == 64)
        pathtrace_impl(a->d, cam, w, h, pixels, pixels ? npix : w * h, frame0, nframes, maxDepth, rr,
                       static_cast<double*>(img), nthreads, ray_counts, static_cast<const ConstantCache<double>*>(nullptr),
                       mode);
    else
        pathtrace_impl(a->f, cam, w, h, pixels, pixels ? npix : w * h, frame0, nframes, maxDepth, rr,
                       static_cast<float*>(img), nthreads, ray_counts, static_cast<const ConstantCache<float>*>(nullptr),
                       mode);
}

// The cached path tracer's estimator with a constant cache (see
// ConstantCache), float: what cupbr_cache_render computes when the network
// answers `value` everywhere.  Russian roulette off.
void ora_pathtrace_cached_f32(void* s, const float* cam, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                              uint32_t maxDepth, uint32_t cache_depth, const float* value, int specular, float* img,
                              int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    const ConstantCache<float> c{cache_depth, V3<float>(value[0], value[1], value[2]), specular != 0};
    pathtrace_impl(a->f, cam, w, h, nullptr, w * h, frame0, nframes, maxDepth, 0, img, nthreads, nullptr, &c);
}

// VOLUME method (VolumeRenderer.cu:214-310) running mean, float.
void ora_volumetrace_f32(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                         uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img, int nthreads,
                         uint64_t* ray_counts);
// VOLUME with the physical estimator (the scene medium's light term carries
// the phase value), float.
void ora_volumetrace_phys_f32(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels,
                              uint32_t npix, uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img,
                              int nthreads, uint64_t* ray_counts);
static void volumetrace_impl(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels,
                             uint32_t npix, uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img,
                             int nthreads, uint64_t* ray_counts, bool physical);
void ora_volumetrace_f32(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t npix,
                         uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img, int nthreads,
                         uint64_t* ray_counts) {
    volumetrace_impl(s, camf, w, h, pixels, npix, frame0, nframes, maxDepth, rr, img, nthreads, ray_counts, false);
}
void ora_volumetrace_phys_f32(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels,
                              uint32_t npix, uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img,
                              int nthreads, uint64_t* ray_counts) {
    volumetrace_impl(s, camf, w, h, pixels, npix, frame0, nframes, maxDepth, rr, img, nthreads, ray_counts, true);
}
static void volumetrace_impl(void* s, const float* camf, uint32_t w, uint32_t h, const uint32_t* pixels,
                             uint32_t npix, uint32_t frame0, uint32_t nframes, uint32_t maxDepth, int rr, float* img,
                             int nthreads, uint64_t* ray_counts, bool physical) {
    AnyScene* a = static_cast<AnyScene*>(s);
    Camera<float> cam = cam_of<float>(camf);
    const int64_t n = pixels ? npix : (int64_t)w * h;
    std::atomic<uint64_t> ext{0}, shd{0};
    parallel_for(n, 16, nthreads, [&](int64_t lo, int64_t hi) {
        RayStats st;
        for (int64_t i = lo; i < hi; ++i) {
            uint32_t tid = pixels ? pixels[i] : (uint32_t)i;
            V3<float> acc(img[3 * i], img[3 * i + 1], img[3 * i + 2]);
            for (uint32_t f = frame0; f < frame0 + nframes; ++f)
                acc = running_mean(acc, trace_volume_path(a->f, cam, tid, w, h, f, maxDepth, rr != 0, &st, physical),
                                   f);
            img[3 * i] = acc.x; img[3 * i + 1] = acc.y; img[3 * i + 2] = acc.z;
        }
        ext += st.extension;
        shd += st.shadow;
    });
    if (ray_counts) { ray_counts[0] = ext.load(); ray_counts[1] = shd.load(); }
}

// GRADIENTDOMAIN frames (gdpt_kernel, GradientDomain.cu:160-246): updates the
// running means of the five w*h*3 images base, gxf, gxb, gyf, gyb (border
// pixels are skipped, as in the reference).
void ora_gdpt_frames(void* s, const float* camf, uint32_t w, uint32_t h, uint32_t frame0, uint32_t nframes,
                     uint32_t maxDepth, float* base, float* gxf, float* gxb, float* gyf, float* gyb, int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    Camera<float> cam = cam_of<float>(camf);
    float* imgs[5] = {base, gxf, gxb, gyf, gyb};
    parallel_for((int64_t)w * h, 16, nthreads, [&](int64_t lo, int64_t hi) {
        for (int64_t p = lo; p < hi; ++p) {
            uint32_t py = (uint32_t)(p / w), px = (uint32_t)(p - (int64_t)w * py);
            if (px == 0 || px == w - 1 || py == 0 || py == h - 1) continue;
            for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
                V3<float> o[5];
                gdpt_pixel(a->f, cam, px, py, w, h, f, maxDepth, o);
                for (int k = 0; k < 5; ++k) {
                    float* q = imgs[k] + 3 * p;
                    V3<float> r = running_mean(V3<float>(q[0], q[1], q[2]), o[k], f);
                    q[0] = r.x; q[1] = r.y; q[2] = r.z;
                }
            }
        }
    });
}

// init_kernel + 50 optimization passes (GradientDomain.cu:248-350, 379-401).
void ora_gdpt_reconstruct(const float* base, const float* gxf, const float* gxb, const float* gyf, const float* gyb,
                          uint32_t w, uint32_t h, float* temp, float* out, float* gx, float* gy, int iterations) {
    gdpt_reconstruct(base, gxf, gxb, gyf, gyb, w, h, temp, out, gx, gy, iterations);
}

// RAYTRACER (RayTracer.cu:11-54) for all w*h pixels.
void ora_raytrace(void* s, const float* camf, uint32_t w, uint32_t h, float* img, int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    Camera<float> cam = cam_of<float>(camf);
    parallel_for((int64_t)w * h, 64, nthreads, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            V3<float> r = raytrace_pixel(a->f, cam, (uint32_t)i, w, h);
            img[3 * i] = r.x; img[3 * i + 1] = r.y; img[3 * i + 2] = r.z;
        }
    });
}

// Density-grid medium (cupbr_b200/csrc/medium.cu restated).  precision 32
// or 64 selects float / double for density, img and the gradients.
//   dims = nx, ny, nz; box = lo.xyz, hi.xyz; mp = majorant, albedo, g, q.
}  // extern "C"
namespace {
template <typename R>
Grid<R> make_grid(const uint32_t* dims, const float* box, const float* mp, const R* density) {
    Grid<R> G;
    G.nx = dims[0];
    G.ny = dims[1];
    G.nz = dims[2];
    G.lo = v3<R>(box);
    G.hi = v3<R>(box + 3);
    G.inv_cell = V3<R>(R(float(G.nx)) / (G.hi.x - G.lo.x), R(float(G.ny)) / (G.hi.y - G.lo.y),
                       R(float(G.nz)) / (G.hi.z - G.lo.z));
    // the reciprocals are formed in float, as the C-ABI does for the kernels
    G.majorant = R(mp[0]);
    G.inv_majorant = R(1.0f / mp[0]);
    G.albedo = R(mp[1]);
    G.g = R(mp[2]);
    G.q = R(mp[3]);
    G.inv_q = R(mp[3] > 0.0f ? 1.0f / mp[3] : 0.0f);
    G.inv_one_minus_q = R(1.0f / (1.0f - mp[3]));
    G.density.assign(density, density + (size_t)G.nx * G.ny * G.nz);
    return G;
}
template <typename R>
void medium_forward_impl(const Scene<R>& sc, const Grid<R>& G, const float* camf, uint32_t w, uint32_t h,
                         const uint32_t* pixels, uint32_t npix, uint32_t spp, uint32_t frame0, uint32_t depth, R* img,
                         int nthreads) {
    const Camera<R> cam = cam_of<R>(camf);
    parallel_for((int64_t)npix, 8, nthreads, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            const uint32_t tid = pixels ? pixels[i] : (uint32_t)i;
            const V3<R> v = medium_pixel(sc, G, cam, tid, w, h, spp, frame0, depth);
            img[3 * i] = v.x;
            img[3 * i + 1] = v.y;
            img[3 * i + 2] = v.z;
        }
    });
}
template <typename R>
void medium_backward_impl(const Scene<R>& sc, const Grid<R>& G, const float* camf, uint32_t w, uint32_t h,
                          uint32_t spp, uint32_t frame0, uint32_t depth, const R* grad_img, R* g_grid, R* g_params,
                          int nthreads) {
    const Camera<R> cam = cam_of<R>(camf);
    const size_t nv = G.density.size(), np = 1 + 6 * sc.objects.size() + 3 * sc.lights.size();
    std::mutex mu;
    parallel_for((int64_t)w * h, 8, nthreads, [&](int64_t lo, int64_t hi) {
        std::vector<R> gg(nv, R(0)), gp(np, R(0));
        for (int64_t i = lo; i < hi; ++i) {
            const V3<R> gi(grad_img[3 * i], grad_img[3 * i + 1], grad_img[3 * i + 2]);
            medium_pixel_adjoint(sc, G, cam, (uint32_t)i, w, h, spp, frame0, depth, gi, gg, gp);
        }
        std::lock_guard<std::mutex> lk(mu);
        for (size_t k = 0; k < nv; ++k) g_grid[k] += gg[k];
        for (size_t k = 0; k < np; ++k) g_params[k] += gp[k];
    });
}
}  // namespace
extern "C" {

void ora_medium_forward(void* s, int precision, const uint32_t* dims, const float* box, const float* mp,
                        const void* density, const float* cam, uint32_t w, uint32_t h, const uint32_t* pixels,
                        uint32_t npix, uint32_t spp, uint32_t frame0, uint32_t depth, void* img, int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    const uint32_t n = pixels ? npix : w * h;
    if (precision == 64)
        medium_forward_impl(a->d, make_grid(dims, box, mp, (const double*)density), cam, w, h, pixels, n, spp, frame0,
                            depth, (double*)img, nthreads);
    else
        medium_forward_impl(a->f, make_grid(dims, box, mp, (const float*)density), cam, w, h, pixels, n, spp, frame0,
                            depth, (float*)img, nthreads);
}
// Adds dLoss/d(density) to g_grid and dLoss/d(params) to g_params
// ([albedo, 3 per object albedo_d, 3 per object albedo_e, 3 per light]) for
// grad_img = dLoss/d(image).
void ora_medium_backward(void* s, int precision, const uint32_t* dims, const float* box, const float* mp,
                         const void* density, const float* cam, uint32_t w, uint32_t h, uint32_t spp, uint32_t frame0,
                         uint32_t depth, const void* grad_img, void* g_grid, void* g_params, int nthreads) {
    AnyScene* a = static_cast<AnyScene*>(s);
    if (precision == 64)
        medium_backward_impl(a->d, make_grid(dims, box, mp, (const double*)density), cam, w, h, spp, frame0, depth,
                             (const double*)grad_img, (double*)g_grid, (double*)g_params, nthreads);
    else
        medium_backward_impl(a->f, make_grid(dims, box, mp, (const float*)density), cam, w, h, spp, frame0, depth,
                             (const float*)grad_img, (float*)g_grid, (float*)g_params, nthreads);
}

// RNG known-answer helpers (FunctionsDetail.h:70-98).
uint32_t ora_tea4(uint32_t a, uint32_t b) { return tea4(a, b); }
void ora_rnd_stream(uint32_t seed, int n, float* out, uint32_t* states) {
    for (int i = 0; i < n; ++i) {
        out[i] = rnd<float>(seed);
        if (states) states[i] = seed;
    }
}

// BSDF sample/eval known answers: one call per (material, seed, inc, n).
void ora_sample_direction(const float* mat, uint32_t seed, const float* inc, const float* n, float* out4,
                          uint32_t* seed_out) {
    Scene<float> tmp;
    float geo[12] = {0};
    add_object(tmp, SPHERE, geo, 1.0f, mat, nullptr, 0, nullptr);
    V4<float> r = sampleDirection(tmp.objects[0].mat, seed, v3<float>(inc), v3<float>(n));
    out4[0] = r.x; out4[1] = r.y; out4[2] = r.z; out4[3] = r.w;
    if (seed_out) *seed_out = seed;
}
void ora_brdf(const float* mat, const float* inc, const float* out, const float* n, float* res3) {
    Scene<float> tmp;
    float geo[12] = {0};
    add_object(tmp, SPHERE, geo, 1.0f, mat, nullptr, 0, nullptr);
    V3<float> r = brdf(tmp.objects[0].mat, v3<float>(inc), v3<float>(out), v3<float>(n));
    res3[0] = r.x; res3[1] = r.y; res3[2] = r.z;
}
void ora_light_sample(const float* l, uint32_t seed, const float* P, float* rad3, float* dir3, float* dist,
                      uint32_t* seed_out) {
    Scene<float> tmp;
    add_light(tmp, l);
    V3<float> dir;
    float d;
    V3<float> r = light_sample(tmp.lights[0], seed, v3<float>(P), dir, d);
    rad3[0] = r.x; rad3[1] = r.y; rad3[2] = r.z;
    dir3[0] = dir.x; dir3[1] = dir.y; dir3[2] = dir.z;
    *dist = d;
    if (seed_out) *seed_out = seed;
}

void ora_tonemap(const float* hdr, uint64_t npix, int type, float exposure, uint8_t* out) {
    parallel_for((int64_t)npix, 4096, 0, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            if (type == 0) reinhard(hdr + 3 * i, exposure, out + 4 * i);
            else gamma(hdr + 3 * i, out + 4 * i);
        }
    });
}
void ora_bloom(const float* hdr, uint32_t w, uint32_t h, const float* th, float* out) { bloom(hdr, w, h, th, out); }

}  // extern "C"
