// Scene commit: reference object order, primitive keys, SAH BVH build and
// device upload.  Compiled with -ffp-contract=off: the host-side precomputed
// values (triangle edges and normals, normalized plane / quad normals, quad
// extents, light normals and areas, albedo_d / pi) are the same single IEEE
// operations the reference performs at construction or per test.
#include "device_scene.hpp"
#include "dev_alloc.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>

#include <cuda_runtime.h>

#include "bvh_gpu.hpp"
#include "env_dist.hpp"
#include "parallel.hpp"

namespace cupbr_b200 {

namespace {

struct V { float x, y, z; };
inline V v3(const float* p) { return {p[0], p[1], p[2]}; }
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V cross(V v, V w) { return {v.y * w.z - v.z * w.y, v.z * w.x - v.x * w.z, v.x * w.y - v.y * w.x}; }
inline float dot(V v, V w) { return v.x * w.x + v.y * w.y + v.z * w.z; }
inline float norm(V v) { return std::sqrt(dot(v, v)); }
inline V normalize(V v) { float n = norm(v); return {v.x / n, v.y / n, v.z / n}; }  // VectorFunctionsDetail.h:55-59

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float ubits(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

struct F4 { float x, y, z, w; };
inline F4 f4(V v, float w) { return {v.x, v.y, v.z, w}; }

inline PrimBox inflate(PrimBox b, float abs_eps) {
    for (int k = 0; k < 3; ++k) {
        float m = std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k]));
        float e = abs_eps + m * (1.0f / 65536.0f);
        b.lo[k] -= e;
        b.hi[k] += e;
    }
    return b;
}

// A host array that is not zero-filled on construction: every element is
// written before it is uploaded (saves a pass over ~100 MB for a 2M-triangle
// scene).
template <typename T>
struct HostArray {
    std::unique_ptr<T[]> p;
    size_t n = 0;
    explicit HostArray(size_t count) : p(count ? new T[count] : nullptr), n(count) {}
    T& operator[](size_t i) { return p[i]; }
    const T* data() const { return p.get(); }
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
};

template <typename Cont, typename T>
bool upload(GpuScene& g, const Cont& v, const T*& out, std::string& err) {
    if (v.empty()) { out = nullptr; return true; }
    void* p = nullptr;
    size_t bytes = v.size() * sizeof(T);
    cudaError_t e = dev_alloc(&p, bytes);
    if (e != cudaSuccess) { err = std::string("cudaMalloc: ") + cudaGetErrorString(e); return false; }
    g.buffers.push_back(p);
    e = cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { err = std::string("cudaMemcpy: ") + cudaGetErrorString(e); return false; }
    g.device_bytes += bytes;
    out = reinterpret_cast<const T*>(p);
    return true;
}

void order_rec(const HostScene& sc, const std::vector<uint32_t>& objs, std::vector<uint32_t>& out) {
    size_t n = objs.size();
    if (n == 0) return;
    auto minx = [&](uint32_t i) {
        const HObject& o = sc.objects[i];
        return o.finite_box ? o.box_lo[0] : -INFINITY;
    };
    if (n == 1) { out.push_back(objs[0]); return; }
    if (n == 2) {  // BoundingVolumeHierarchy.cpp:65-89
        if (minx(objs[0]) < minx(objs[1])) { out.push_back(objs[0]); out.push_back(objs[1]); }
        else { out.push_back(objs[1]); out.push_back(objs[0]); }
        return;
    }
    std::vector<size_t> idx(n);  // :90-122: stable sort by box min along x, split at n/2
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return minx(objs[a]) < minx(objs[b]); });
    size_t mid = n / 2;
    std::vector<uint32_t> l, r;
    l.reserve(mid);
    r.reserve(n - mid);
    for (size_t i = 0; i < n; ++i) (i < mid ? l : r).push_back(objs[idx[i]]);
    order_rec(sc, l, out);
    order_rec(sc, r, out);
}

}  // namespace

GpuScene::~GpuScene() { release(); }

void GpuScene::release() {
    for (void* p : buffers) cudaFree(p);
    buffers.clear();
    dev = DeviceScene{};
    device_bytes = 0;
    committed = false;
}

// The reference splits on axis (rand() / RAND_MAX) % 3, which is 0 unless
// rand() returns exactly RAND_MAX, so the split axis is x.
std::vector<uint32_t> reference_object_order(const HostScene& sc) {
    std::vector<uint32_t> all(sc.objects.size()), out;
    std::iota(all.begin(), all.end(), 0u);
    out.reserve(all.size());
    order_rec(sc, all, out);
    return out;
}

DMaterial device_material(const HMaterial& m) {
    DMaterial d;
    const float pi = static_cast<float>(M_PI);
    d.e = make_float4(m.albedo_e[0], m.albedo_e[1], m.albedo_e[2], (float)m.type);
    d.d = make_float4(m.albedo_d[0], m.albedo_d[1], m.albedo_d[2], m.shininess);
    d.s = make_float4(m.albedo_s[0], m.albedo_s[1], m.albedo_s[2], m.roughness);
    d.dl = make_float4(m.albedo_d[0] / pi, m.albedo_d[1] / pi, m.albedo_d[2] / pi, m.eta);  // MaterialDetail.h:202-207
    d.ss = make_float4(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2], m.g);
    d.sa = make_float4(m.sigma_a[0], m.sigma_a[1], m.sigma_a[2], m.interface_glass ? 1.0f : 0.0f);
    return d;
}

bool commit_scene(GpuScene& g, const BvhBuildParams& params, std::string& err) {
    const auto t_commit = std::chrono::steady_clock::now();
    g.release();
    g.params = params;
    ++g.generation;
    const HostScene& sc = g.host;
    const size_t nobj = sc.objects.size();

    // primitive keys in the reference's object order
    g.dfs_order = reference_object_order(sc);
    g.key_base.assign(nobj, 0);
    uint32_t nkeys = 0;
    for (uint32_t o : g.dfs_order) {
        g.key_base[o] = nkeys;
        const HObject& ob = sc.objects[o];
        nkeys += (ob.type == GEO_MESH || ob.type == GEO_TRIANGLE) ? ob.tri_count : 1u;
    }
    g.key_obj.assign(nkeys, -1);

    // scene-wide absolute inflation: a few ulps of the largest coordinate
    float maxabs = 1.0f;
    {
        const int64_t nv = (int64_t)sc.tri_verts.size(), grain = 1 << 18;
        std::vector<float> part((size_t)(nv / grain + 1), 0.0f);
        parallel_for(nv, grain, [&](int64_t lo, int64_t hi) {
            float m = 0.0f;
            for (int64_t i = lo; i < hi; ++i) m = std::max(m, std::fabs(sc.tri_verts[i]));
            part[(size_t)(lo / grain)] = m;
        });
        for (float m : part) maxabs = std::max(maxabs, m);
    }
    for (const HObject& ob : sc.objects)
        for (int k = 0; k < 3; ++k) maxabs = std::max(maxabs, std::fabs(ob.p0[k]) + std::fabs(ob.radius));
    const float abs_eps = maxabs * (1.0f / 65536.0f);

    // triangles in object order (object o's run starts at tri_off[o])
    std::vector<uint32_t> sph_obj, quad_obj_ids, plane_obj, mesh_obj;
    std::vector<size_t> tri_off(nobj, 0);
    size_t nT = 0;
    for (uint32_t o = 0; o < nobj; ++o) {
        const HObject& ob = sc.objects[o];
        switch (ob.type) {
            case GEO_MESH:
            case GEO_TRIANGLE: mesh_obj.push_back(o); tri_off[o] = nT; nT += ob.tri_count; break;
            case GEO_SPHERE: sph_obj.push_back(o); g.key_obj[g.key_base[o]] = (int32_t)o; break;
            case GEO_QUAD: quad_obj_ids.push_back(o); g.key_obj[g.key_base[o]] = (int32_t)o; break;
            case GEO_PLANE: plane_obj.push_back(o); g.key_obj[g.key_base[o]] = (int32_t)o; break;
        }
    }
    HostArray<uint32_t> tri_obj(nT), tri_gid(nT);
    parallel_for((int64_t)mesh_obj.size(), 1, [&](int64_t lo, int64_t hi) {
        for (int64_t m = lo; m < hi; ++m) {
            const uint32_t o = mesh_obj[(size_t)m];
            const HObject& ob = sc.objects[o];
            const size_t b = tri_off[o];
            for (uint32_t t = 0; t < ob.tri_count; ++t) {
                tri_obj[b + t] = o;
                tri_gid[b + t] = ob.tri_begin + t;
                g.key_obj[g.key_base[o] + t] = (int32_t)o;
            }
        }
    });
    const size_t nS = sph_obj.size(), nQ = quad_obj_ids.size(), nP = plane_obj.size();
    if (nT + nS + nQ >= (1u << 28)) { err = "too many primitives (limit 2^28)"; return false; }

    std::vector<PrimBox> boxes[3];
    boxes[0].resize(nT);
    parallel_for((int64_t)nT, 16384, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            const float* t = &sc.tri_verts[9 * (size_t)tri_gid[i]];
            PrimBox b;
            for (int k = 0; k < 3; ++k) {
                b.lo[k] = std::min(t[k], std::min(t[3 + k], t[6 + k]));
                b.hi[k] = std::max(t[k], std::max(t[3 + k], t[6 + k]));
            }
            boxes[0][i] = inflate(b, abs_eps);
        }
    });
    boxes[1].resize(nS);
    for (size_t i = 0; i < nS; ++i) {
        const HObject& ob = sc.objects[sph_obj[i]];
        PrimBox b;
        for (int k = 0; k < 3; ++k) { b.lo[k] = ob.p0[k] - ob.radius; b.hi[k] = ob.p0[k] + ob.radius; }
        boxes[1][i] = inflate(b, abs_eps);
    }
    std::vector<V> qn(nQ);
    boxes[2].resize(nQ);
    for (size_t i = 0; i < nQ; ++i) {
        const HObject& ob = sc.objects[quad_obj_ids[i]];
        V n = normalize(v3(ob.p1));  // QuadDetail.h:12 constructor normalizes
        qn[i] = n;
        // corners: n.r = 0, e1.r = +-|e1|^2, e2.r = +-|e2|^2  (r = I - position)
        double M[3][3] = {{n.x, n.y, n.z}, {ob.p2[0], ob.p2[1], ob.p2[2]}, {ob.p3[0], ob.p3[1], ob.p3[2]}};
        double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        double s1 = (double)ob.p2[0] * ob.p2[0] + (double)ob.p2[1] * ob.p2[1] + (double)ob.p2[2] * ob.p2[2];
        double s2 = (double)ob.p3[0] * ob.p3[0] + (double)ob.p3[1] * ob.p3[1] + (double)ob.p3[2] * ob.p3[2];
        PrimBox b;
        if (std::fabs(det) < 1e-12 * std::sqrt(s1 * s2) || s1 == 0.0 || s2 == 0.0) {
            for (int k = 0; k < 3; ++k) { b.lo[k] = -1e30f; b.hi[k] = 1e30f; }
        } else {
            for (int k = 0; k < 3; ++k) { b.lo[k] = INFINITY; b.hi[k] = -INFINITY; }
            for (int c = 0; c < 4; ++c) {
                double rhs[3] = {0.0, (c & 1) ? s1 : -s1, (c & 2) ? s2 : -s2};
                double r[3];
                for (int col = 0; col < 3; ++col) {  // Cramer's rule
                    double A[3][3];
                    std::memcpy(A, M, sizeof A);
                    for (int row = 0; row < 3; ++row) A[row][col] = rhs[row];
                    double dd = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                                A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                                A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
                    r[col] = dd / det;
                }
                for (int k = 0; k < 3; ++k) {
                    float v = (float)(ob.p0[k] + r[k]);
                    b.lo[k] = std::min(b.lo[k], v);
                    b.hi[k] = std::max(b.hi[k], v);
                }
            }
            for (int k = 0; k < 3; ++k) {  // corners were rounded once more
                float e = 1e-6f * (std::fabs(b.lo[k]) + std::fabs(b.hi[k]));
                b.lo[k] -= e;
                b.hi[k] += e;
            }
        }
        boxes[2][i] = inflate(b, abs_eps);
    }

    uint32_t offs[3] = {0u, (uint32_t)nT, (uint32_t)(nT + nS)};
    std::vector<uint32_t> perm[3];
    float4* dev_nodes = nullptr;  // device build: the node array is already on the GPU
    uint32_t dev_n_nodes = 0;
    const auto t_bvh = std::chrono::steady_clock::now();
    g.bvh_device = params.device;
    if (params.device) {
        if (!build_bvh_device(boxes, 3, offs, params, perm, g.bvh, &dev_nodes, &dev_n_nodes, 0, err)) return false;
        g.buffers.push_back(dev_nodes);
        g.device_bytes += (uint64_t)dev_n_nodes * BVH_NODE_BYTES;
    } else {
        build_bvh(boxes, 3, offs, params, perm, g.bvh);
    }
    g.bvh_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_bvh).count();
    // A 4-wide traversal pushes at most 3 entries per level of the path it is
    // on, and the culled entries are popped first, so in practice the stack
    // stays far below 3 x depth; an overflow is still counted on the device
    // (the renderers' error count) rather than ruled out here.  A tree whose
    // single path is longer than the stack is rejected.
    if (g.bvh.stats.max_depth + 2 > 64) {
        err = "BVH deeper than the traversal stack (" + std::to_string(g.bvh.stats.max_depth) + ")";
        return false;
    }

    // triangle slots: (v1, key), (v2 - v1, obj), (v3 - v1, 0); normals (TriangleDetail.h:11-19)
    HostArray<F4> tris(3 * nT), trin(nT);
    parallel_for((int64_t)nT, 16384, [&](int64_t lo, int64_t hi) {
        for (int64_t s = lo; s < hi; ++s) {
            uint32_t i = perm[0][s];
            const float* t = &sc.tri_verts[9 * (size_t)tri_gid[i]];
            V a = v3(t), b = v3(t + 3), c = v3(t + 6);
            V e1 = sub(b, a), e2 = sub(c, a);
            uint32_t o = tri_obj[i];
            uint32_t key = g.key_base[o] + (tri_gid[i] - sc.objects[o].tri_begin);
            tris[3 * s + 0] = f4(a, ubits(key));
            tris[3 * s + 1] = f4(e1, ubits(o));
            tris[3 * s + 2] = f4(e2, 0.0f);
            trin[s] = f4(normalize(cross(e1, e2)), 0.0f);  // TriangleDetail.h:16
        }
    });
    std::vector<F4> sph(2 * nS);
    for (size_t s = 0; s < nS; ++s) {
        uint32_t o = sph_obj[perm[1][s]];
        const HObject& ob = sc.objects[o];
        sph[2 * s] = f4(v3(ob.p0), ubits(g.key_base[o]));
        sph[2 * s + 1] = {ob.radius, ob.radius * ob.radius, ubits(o), 0.0f};
    }
    std::vector<F4> quads(4 * nQ);
    std::vector<int32_t> qobj(nQ);
    for (size_t s = 0; s < nQ; ++s) {
        uint32_t qi = perm[2][s];
        uint32_t o = quad_obj_ids[qi];
        const HObject& ob = sc.objects[o];
        V n = qn[qi], p = v3(ob.p0), e1 = v3(ob.p2), e2 = v3(ob.p3);
        quads[4 * s + 0] = f4(p, ubits(g.key_base[o]));
        quads[4 * s + 1] = f4(n, dot(p, n));
        quads[4 * s + 2] = f4(e1, dot(e1, e1));
        quads[4 * s + 3] = f4(e2, dot(e2, e2));
        qobj[s] = (int32_t)o;
    }
    std::vector<F4> planes(2 * nP);
    for (size_t s = 0; s < nP; ++s) {
        uint32_t o = plane_obj[s];
        const HObject& ob = sc.objects[o];
        planes[2 * s] = f4(v3(ob.p0), ubits(g.key_base[o]));
        planes[2 * s + 1] = f4(normalize(v3(ob.p1)), ubits(o));  // PlaneDetail.h:12
    }
    std::vector<DObject> objs(nobj);
    std::vector<DMaterial> mats(nobj);
    for (size_t o = 0; o < nobj; ++o) {
        const HObject& ob = sc.objects[o];
        objs[o].lo = make_float4(ob.box_lo[0], ob.box_lo[1], ob.box_lo[2], ob.finite_box ? 1.0f : 0.0f);
        objs[o].hi = make_float4(ob.box_hi[0], ob.box_hi[1], ob.box_hi[2], ubits((uint32_t)o));
        mats[o] = device_material(ob.mat);
    }
    std::vector<DLight> lights(sc.lights.size());
    for (size_t i = 0; i < sc.lights.size(); ++i) {
        const HLight& l = sc.lights[i];
        V e1 = v3(l.he1), e2 = v3(l.he2);
        float area = 4.0f * norm(e1) * norm(e2);  // LightDetail.h:40-41
        V n = normalize(cross(e1, e2));
        lights[i].pos = make_float4(l.position[0], l.position[1], l.position[2], (float)l.type);
        lights[i].I = make_float4(l.intensity[0], l.intensity[1], l.intensity[2], 0.0f);
        lights[i].L = make_float4(l.radiance[0], l.radiance[1], l.radiance[2], area);
        lights[i].e1 = make_float4(e1.x, e1.y, e1.z, 0.0f);
        lights[i].e2 = make_float4(e2.x, e2.y, e2.z, 0.0f);
        lights[i].n = make_float4(n.x, n.y, n.z, 0.0f);
    }
    // single-object traces (TracingDetail.h:68-116): per object its type and
    // key range, per key the slot of its primitive
    std::vector<int4> oinfo(nobj);
    std::vector<uint32_t> kslot(nkeys, 0u);
    for (size_t o = 0; o < nobj; ++o) {
        const HObject& ob = sc.objects[o];
        uint32_t cnt = (ob.type == GEO_MESH || ob.type == GEO_TRIANGLE) ? ob.tri_count : 1u;
        oinfo[o] = make_int4(ob.type, (int)g.key_base[o], (int)cnt, 0);
    }
    parallel_for((int64_t)nT, 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t s = lo; s < hi; ++s) {
            const uint32_t i = perm[0][s];
            const uint32_t o = tri_obj[i];
            kslot[g.key_base[o] + (tri_gid[i] - sc.objects[o].tri_begin)] = (uint32_t)s;
        }
    });
    for (size_t s = 0; s < nS; ++s) kslot[g.key_base[sph_obj[perm[1][s]]]] = (uint32_t)s;
    for (size_t s = 0; s < nQ; ++s) kslot[g.key_base[quad_obj_ids[perm[2][s]]]] = (uint32_t)s;
    for (size_t s = 0; s < nP; ++s) kslot[g.key_base[plane_obj[s]]] = (uint32_t)s;
    HostArray<F4> env((size_t)sc.env_w * sc.env_h);
    parallel_for((int64_t)env.size(), 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) env[i] = {sc.env[3 * i], sc.env[3 * i + 1], sc.env[3 * i + 2], 0.0f};
    });

    DeviceScene& D = g.dev;
    const F4* p;
    if (dev_nodes) {
        D.nodes = dev_nodes;
        D.n_nodes = dev_n_nodes;
    } else {
        std::vector<F4> nodes(g.bvh.nodes.size() / 4);
        std::memcpy(nodes.data(), g.bvh.nodes.data(), g.bvh.nodes.size() * sizeof(float));
        if (!upload(g, nodes, p, err)) return false;
        D.nodes = reinterpret_cast<const float4*>(p);
        D.n_nodes = (uint32_t)(nodes.size() / BVH_NODE_F4);  // nodes, not float4s
    }
    if (!upload(g, tris, p, err)) return false;
    D.tris = reinterpret_cast<const float4*>(p);
    if (!upload(g, trin, p, err)) return false;
    D.tri_n = reinterpret_cast<const float4*>(p);
    if (!upload(g, sph, p, err)) return false;
    D.spheres = reinterpret_cast<const float4*>(p);
    if (!upload(g, quads, p, err)) return false;
    D.quads = reinterpret_cast<const float4*>(p);
    const int32_t* qo;
    if (!upload(g, qobj, qo, err)) return false;
    D.quad_obj = qo;
    if (!upload(g, planes, p, err)) return false;
    D.planes = reinterpret_cast<const float4*>(p);
    const DObject* dobj;
    if (!upload(g, objs, dobj, err)) return false;
    D.objects = dobj;
    const DMaterial* dmat;
    if (!upload(g, mats, dmat, err)) return false;
    D.materials = dmat;
    const DLight* dl;
    if (!upload(g, lights, dl, err)) return false;
    D.lights = dl;
    if (!upload(g, env, p, err)) return false;
    D.env = reinterpret_cast<const float4*>(p);
    D.tex = nullptr;
    D.obj_tex = nullptr;
    D.tex_w = D.tex_h = 0;
    if (sc.tex_w && sc.tex_h) {
        HostArray<F4> tex((size_t)sc.tex_w * sc.tex_h);
        parallel_for((int64_t)tex.size(), 65536, [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; ++i) tex[i] = {sc.tex[3 * i], sc.tex[3 * i + 1], sc.tex[3 * i + 2], 0.0f};
        });
        if (!upload(g, tex, p, err)) return false;
        D.tex = const_cast<float4*>(reinterpret_cast<const float4*>(p));
        std::vector<F4> ot(3 * nobj, F4{0.0f, 0.0f, 0.0f, 0.0f});
        for (size_t o = 0; o < nobj; ++o) {
            const HObject& ob = sc.objects[o];
            if (!ob.textured) continue;
            const float uu = ob.tex_u[0] * ob.tex_u[0] + ob.tex_u[1] * ob.tex_u[1] + ob.tex_u[2] * ob.tex_u[2];
            const float vv = ob.tex_v[0] * ob.tex_v[0] + ob.tex_v[1] * ob.tex_v[1] + ob.tex_v[2] * ob.tex_v[2];
            ot[3 * o] = {ob.tex_origin[0], ob.tex_origin[1], ob.tex_origin[2], 1.0f};
            ot[3 * o + 1] = {ob.tex_u[0] / uu, ob.tex_u[1] / uu, ob.tex_u[2] / uu, 0.0f};
            ot[3 * o + 2] = {ob.tex_v[0] / vv, ob.tex_v[1] / vv, ob.tex_v[2] / vv, 0.0f};
        }
        if (!upload(g, ot, p, err)) return false;
        D.obj_tex = reinterpret_cast<const float4*>(p);
        D.tex_w = sc.tex_w;
        D.tex_h = sc.tex_h;
    }
    {
        const EnvDistribution ed = build_env_distribution(sc.env.data(), sc.env_w, sc.env_h);
        const float* t;
        if (!upload(g, ed.marg, t, err)) return false;
        D.env_marg = t;
        if (!upload(g, ed.cond, t, err)) return false;
        D.env_cond = t;
        if (!upload(g, ed.pdf, t, err)) return false;
        D.env_pdf = t;
        if (!upload(g, ed.cosb, t, err)) return false;
        D.env_cosb = t;
        D.env_cw = ed.cw;
        D.env_ch = ed.ch;
    }
    const int4* oi;
    if (!upload(g, oinfo, oi, err)) return false;
    D.obj_info = oi;
    const uint32_t* ks;
    if (!upload(g, kslot, ks, err)) return false;
    D.key_slot = ks;
    D.n_tris = (uint32_t)nT;
    D.n_spheres = (uint32_t)nS;
    D.n_quads = (uint32_t)nQ;
    D.n_planes = (uint32_t)nP;
    D.n_objects = (uint32_t)nobj;
    D.n_lights = (uint32_t)sc.lights.size();
    D.env_w = sc.env_w;
    D.env_h = sc.env_h;
    D.sphere_base = (uint32_t)nT;
    D.quad_base = (uint32_t)(nT + nS);
    D.vol_sigma_s = make_float4(sc.vol_sigma_s[0], sc.vol_sigma_s[1], sc.vol_sigma_s[2], sc.vol_g);
    D.vol_sigma_a = make_float4(sc.vol_sigma_a[0], sc.vol_sigma_a[1], sc.vol_sigma_a[2], 0.0f);
    g.committed = true;
    g.commit_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_commit).count();
    return true;
}

}  // namespace cupbr_b200
